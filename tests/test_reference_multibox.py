"""multi_dielectric_box3d cases of the reference's suite (test/shape/multi_box3d.jl:229-358)
on the library's mesher: a single box equals single_dielectric_box3d; touching boxes share
their common face once, with (eps of the box the normal leaves, eps of the other) on it, and
the quadrature weights integrate the exposed plus shared area; a two-box system solves with
finite sigma. Also the corner-pair discovery case of build_neighbor_list. No GPU except
the solve."""
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


@pytest.mark.gpu
def test_two_box_solver_integration(bie):
    itf = bie.multi_dielectric_box3d(4, 0.3, [box((0.0, 0.0, 0.0), (1, 1, 1)), box((1.0, 0.0, 0.0), (1, 1, 1))],
                                     [2.0, 4.0], 1.0)
    op = bie.lhs_dielectric_box3d(itf)
    rhs = bie.rhs_dielectric_box3d(itf, bie.PointSource((3.0, 0.0, 0.0), 1.0), 1.0)
    assert op.shape == (itf.n, itf.n) and rhs.shape == (itf.n,)
    sigma, st = bie.gpu_solve(op, rhs, rtol=1e-10, precision="fp64")
    assert sigma.shape == (itf.n,) and np.all(np.isfinite(sigma)) and st.solved


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
