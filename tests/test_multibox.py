"""Multi-material geometry (multi_dielectric_box3d, src/shape/box3d_multi.jl:358-386): two
separated boxes with different eps_in. The plain FP64 GPU solve matches the oracle's dense
LU of D^T + C + diag(t_P) to 1e-12, with and without the diagonal right preconditioner
(dielectric_diagonal_scaling, src/solver/multi_rhs.jl:234-247); the refined solves
(FP32 for few columns, split-BF16 tensor cores for 8 or more) to 1e-8."""
import numpy as np
import pytest
import scipy.linalg as sla

pytestmark = pytest.mark.gpu

CENTERS = [(-0.45, 0.0, 0.0), (0.45, 0.05, 0.0)]
DIMS = [(0.6, 0.5, 0.4), (0.5, 0.6, 0.5)]
EPS = [4.0, 12.0]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def two_boxes(bie, orc):
    boxes = [{"center": c, "Lx": d[0], "Ly": d[1], "Lz": d[2]} for c, d in zip(CENTERS, DIMS)]
    itf = bie.multi_dielectric_box3d(4, 0.15, boxes, EPS, 1.0)
    m = orc.Mesh.multi_box(4, 0.15, CENTERS, DIMS, EPS, 1.0)
    assert itf.n == m.n
    ups, adp = orc.build_neighbor_list(m, 8, 1e-9, True)
    Cm = orc.DT_corrections(m, ups, adp, 1e-9)
    A = m.DT_dense(with_diag=True) + Cm.toarray()
    rng = np.random.default_rng(8)
    # sources inside either box (eps_src = that box's eps_in), 10 right-hand sides
    cols = []
    for c in range(10):
        b = c % 2
        p = np.array(CENTERS[b]) + rng.uniform(-0.3, 0.3, 3) * np.array(DIMS[b])
        cols.append((tuple(p), float(rng.standard_normal()), EPS[b]))
    B = np.stack([orc.rhs_point(m.pts, m.nrm, p, q, e) for p, q, e in cols], axis=1)
    X = sla.lu_solve(sla.lu_factor(A), B)
    F = np.stack([bie.rhs_dielectric_box3d(itf, bie.PointSource(p, q), e) for p, q, e in cols], axis=1)
    assert rel(F, B) < 1e-14
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    return itf, op, B, X


@pytest.mark.parametrize("precondition", [False, True])
def test_plain_fp64_vs_lu(bie, two_boxes, precondition):
    itf, op, B, X = two_boxes
    S, st = bie.gpu_solve(op, B, rtol=1e-14, itmax=600, precision="fp64", precondition=precondition)
    for c in range(B.shape[1]):
        assert rel(S[:, c], X[:, c]) < 1e-12, c


@pytest.mark.parametrize("k,precision", [(3, "bf16x3"), (10, "bf16x3"), (10, "fp32")])
def test_refined_vs_lu(bie, two_boxes, k, precision):
    itf, op, B, X = two_boxes
    S, st = bie.gpu_solve(op, B[:, :k], rtol=1e-11, itmax=600, precision=precision, precondition=True)
    assert st.solved and st.lowp_matvecs > 0
    for c in range(k):
        assert rel(S[:, c], X[:, c]) < 1e-8, c


def test_preconditioner_is_inverse_contrast(bie, two_boxes):
    itf = two_boxes[0]
    p = bie.dielectric_diagonal_scaling(itf)
    assert np.allclose(p * itf.diag, 1.0, rtol=1e-15, atol=0)
    assert len(np.unique(np.round(p, 12))) == 2  # one value per material
