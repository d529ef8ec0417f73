"""multi_dielectric_box3d cases of the reference's suite (test/shape/multi_box3d.jl:229-358)
on the library's mesher: a single box equals single_dielectric_box3d; touching boxes share
their common face once, with (eps of the box the normal leaves, eps of the other) on it, and
the quadrature weights integrate the exposed plus shared area. Two touching cubes: set-up
equal to the oracle's, and the plain FP64 GPU solve against the oracle's dense LU of
D^T + C + diag(t_P) to 1e-12 (refined: 1e-8). Also the corner-pair discovery case of
build_neighbor_list. No GPU except the solves."""
import numpy as np
import pytest


def box(center, L):
    return {"center": center, "Lx": L[0], "Ly": L[1], "Lz": L[2]}


def eps_pairs(itf):
    return {(float(a), float(b)) for a, b in zip(itf.eps_in, itf.eps_out)}


def test_single_box_equivalence(bie):
    single = bie.single_dielectric_box3d(1.0, 1.0, 1.0, 4, 0.3, 2.0, 1.0)
    multi = bie.multi_dielectric_box3d(4, 0.3, [box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))], [2.0], 1.0)
    assert multi.npanels == single.npanels and multi.n == single.n
    assert np.all(multi.eps_in == 2.0) and np.all(multi.eps_out == 1.0)


def test_two_touching_boxes(bie):
    itf = bie.multi_dielectric_box3d(4, 0.3, [box((0.0, 0.0, 0.0), (1, 1, 1)), box((1.0, 0.0, 0.0), (1, 1, 1))],
                                     [2.0, 4.0], 1.0)
    assert itf.npanels > 0 and itf.n > 0
    assert {(2.0, 1.0), (4.0, 1.0), (4.0, 2.0)} <= eps_pairs(itf)
    assert abs(itf.weights.sum() - 11.0) < 0.01


def test_three_boxes_l_shape(bie):
    itf = bie.multi_dielectric_box3d(4, 0.3, [box((0.0, 0.0, 0.0), (1, 1, 1)), box((1.0, 0.0, 0.0), (1, 1, 1)),
                                              box((0.0, 1.0, 0.0), (1, 1, 1))], [2.0, 3.0, 4.0])
    assert itf.npanels > 0
    assert abs(itf.weights.sum() - 16.0) < 0.01


def test_different_sized_touching_boxes(bie):
    itf = bie.multi_dielectric_box3d(4, 0.3, [box((0.0, 0.0, 0.0), (2, 2, 2)), box((1.5, 0.0, 0.0), (1, 1, 1))],
                                     [2.0, 4.0], 1.0)
    assert itf.npanels > 0
    assert abs(itf.weights.sum() - 29.0) < 0.1
    assert {(2.0, 1.0), (4.0, 1.0), (4.0, 2.0)} <= eps_pairs(itf)


TOUCH_CENTERS = [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0)]
TOUCH_DIMS = [(1.0, 1.0, 1.0), (1.0, 1.0, 1.0)]
TOUCH_EPS = [2.0, 4.0]


def touching(bie):
    return bie.multi_dielectric_box3d(4, 0.3, [box(c, d) for c, d in zip(TOUCH_CENTERS, TOUCH_DIMS)], TOUCH_EPS, 1.0)


def test_touching_boxes_setup_matches_oracle(bie, orc):
    """Two touching cubes (shared face x = 0.5, _detect_shared_faces_3d and
    _multi_box3d_face_regions, src/shape/box3d_multi.jl:139-356): the library's mesh equals
    the oracle's bit for bit (nodes, normals, weights, per-panel eps pairs, diagonal), the
    neighbour lists are identical and the correction blocks agree to the FP64 rounding level."""
    itf = touching(bie)
    m = orc.Mesh.multi_box(4, 0.3, TOUCH_CENTERS, TOUCH_DIMS, TOUCH_EPS, 1.0)
    assert itf.n == m.n == 2816
    for a, b in ((itf.points, m.pts), (itf.normals, m.nrm), (itf.weights, m.w), (itf.eps_in, m.eps_in),
                 (itf.eps_out, m.eps_out), (itf.is_edge, m.is_edge), (itf.diag, m.diag())):
        assert np.array_equal(a, b)
    ups, adp = bie.build_neighbor_list(itf, 8, 1e-9, correct_edges=True)
    ups_o, adp_o = orc.build_neighbor_list(m, 8, 1e-9, True)
    assert ups == ups_o and sorted(adp) == sorted(adp_o)
    C_lib = bie.laplace3d_DT_corrections(itf, max_order=8, up_tol=1e-9, correct_edges=True).tocsr()
    C_orc = orc.DT_corrections(m, ups_o, adp_o, 1e-9).tocsr()
    assert np.abs((C_lib - C_orc).toarray()).max() <= 1e-13 * np.abs(C_orc.toarray()).max()


@pytest.fixture(scope="module")
def touching_system(bie, orc):
    """O-corr oracle on the touching cubes: dense D^T + C + diag(t_P) and its LU solutions
    for a source outside both boxes (eps_src = eps_out) and one inside each box."""
    import scipy.linalg as sla
    m = orc.Mesh.multi_box(4, 0.3, TOUCH_CENTERS, TOUCH_DIMS, TOUCH_EPS, 1.0)
    ups, adp = orc.build_neighbor_list(m, 8, 1e-9, True)
    A = m.DT_dense(with_diag=True) + orc.DT_corrections(m, ups, adp, 1e-9).toarray()
    cols = [((3.0, 0.0, 0.0), 1.0, 1.0), ((-0.1, 0.2, -0.15), -0.7, 2.0), ((1.2, -0.1, 0.25), 1.3, 4.0)]
    B = np.stack([orc.rhs_point(m.pts, m.nrm, p, q, e) for p, q, e in cols], axis=1)
    X = sla.lu_solve(sla.lu_factor(A), B)
    itf = touching(bie)
    F = np.stack([bie.rhs_dielectric_box3d(itf, bie.PointSource(p, q), e) for p, q, e in cols], axis=1)
    assert np.linalg.norm(F - B) <= 1e-14 * np.linalg.norm(B)
    return itf, B, X


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("precondition", [False, True])
def test_touching_boxes_plain_fp64_vs_lu(bie, touching_system, precondition):
    """Plain FP64 GPU solve of the touching cubes (shared face with the (4, 2) eps pair) against
    the oracle's dense LU to 1e-12 per column; the total polarisation charge of the outside
    source's solution is 0 (no net charge enclosed)."""
    itf, B, X = touching_system
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    assert op.shape == (itf.n, itf.n)
    S, st = bie.gpu_solve(op, B, rtol=1e-14, itmax=600, precision="fp64", precondition=precondition)
    for c in range(B.shape[1]):
        assert rel(S[:, c], X[:, c]) < 1e-12, c
    assert abs(np.dot(itf.weights, S[:, 0])) < 0.1


@pytest.mark.gpu
def test_touching_boxes_refined_vs_lu(bie, touching_system):
    itf, B, X = touching_system
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    S, st = bie.gpu_solve(op, B, rtol=1e-11, itmax=600, precision="fp32", precondition=True)
    assert st.solved and st.lowp_matvecs > 0
    for c in range(B.shape[1]):
        assert rel(S[:, c], X[:, c]) < 1e-8, c


def test_corner_pair_discovery(bie, orc):
    """build_neighbor_list corner-pair discovery (test/kernel/laplace3d_near_corner_pairs.jl):
    two perpendicular n_quad = 3 panels sharing an edge, whose Gauss nodes are all interior,
    form a touching (adaptive) pair exactly when correct_edges is set; library and oracle."""
    ns, ws = bie.gausslegendre(3)
    pa = bie.rect_panel3d_discretize((-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0),
                                     ns, ws, (0.0, 0.0, 1.0))
    pb = bie.rect_panel3d_discretize((0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (0.5, 0.5, 1.0), (0.5, -0.5, 1.0),
                                     ns, ws, (1.0, 0.0, 0.0))
    itf = bie.DielectricInterface([pa, pb], [1.0, 1.0], [1.0, 1.0])
    _, adaptive = bie.build_neighbor_list(itf, 8, 1e-6, correct_edges=False)
    assert not adaptive
    itf2 = bie.DielectricInterface([pa, pb], [1.0, 1.0], [1.0, 1.0])
    _, adaptive = bie.build_neighbor_list(itf2, 8, 1e-6, correct_edges=True)
    assert (0, 1) in adaptive or (1, 0) in adaptive
    m = orc.Mesh.from_panels(3, [itf.corners[0], itf.corners[1]], [[0, 0, 1], [1, 0, 0]])
    assert not orc.build_neighbor_list(m, 8, 1e-6, False)[1]
    adp = orc.build_neighbor_list(m, 8, 1e-6, True)[1]
    assert set(map(tuple, adp)) & {(0, 1), (1, 0)}
