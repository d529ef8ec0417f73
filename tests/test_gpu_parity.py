"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (relative 2-norm unless stated):
  FP64 matvec vs oracle direct sum ........ 1e-13
  FP64 solve sigma vs oracle LU ........... 1e-12   (north-star plain-path bar)
  refined (FP32 / BF16x3) sigma vs oracle . 1e-8    (north-star refined-path bar)
  FP32 matvec vs FP64 matvec .............. 1e-5
"""
import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope="module")
def cfg1(bie, orc):
    itf = bie.single_dielectric_box3d(*CFG1)
    m = orc.Mesh.single_box(*CFG1)
    ups, adp = orc.build_neighbor_list(m, 8, 1e-9, True)
    Cm = orc.DT_corrections(m, ups, adp, 1e-9)
    A = m.DT_dense(with_diag=True)
    return itf, m, Cm, A


def test_matvec_fp64_uncorrected(bie, orc, cfg1, rng):
    itf, m, Cm, A = cfg1
    op = bie.lhs_dielectric_box3d(itf)
    x = rng.standard_normal(itf.n)
    assert rel(op @ x, A @ x) < 1e-13
    X = rng.standard_normal((itf.n, 5))
    Y = op @ X
    for c in range(5):
        assert rel(Y[:, c], A @ X[:, c]) < 1e-13


def test_matvec_fp64_corrected(bie, orc, cfg1, rng):
    itf, m, Cm, A = cfg1
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    x = np.cos(0.2 * np.arange(1, itf.n + 1))
    ref = A @ x + Cm @ x
    assert rel(op @ x, ref) < 1e-13
    # the oracle's matrix-free operator agrees with the dense assembly
    assert rel(orc.op_apply(m, x, Cm), ref) < 1e-13


def test_matvec_many_rhs_columnwise(bie, cfg1, rng):
    itf = cfg1[0]
    op = bie.batched_lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-9, 1e-9, 8)
    X = rng.standard_normal((itf.n, 70))  # exercises the 64 + 4 + 2 column chunking
    Y = op @ X
    for c in (0, 17, 63, 64, 69):
        assert np.max(np.abs(Y[:, c] - op @ X[:, c])) < 1e-12


def test_matvec_fp32_close_to_fp64(bie, cfg1, rng):
    itf = cfg1[0]
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-9, 1e-9, 8)
    X = rng.standard_normal((itf.n, 3))
    assert rel(op.mul(X, precision="fp32"), op.mul(X)) < 1e-5


def test_rhs_point_matches_oracle(bie, orc, cfg1):
    itf, m = cfg1[0], cfg1[1]
    f = bie.rhs_dielectric_box3d(itf, bie.PointSource((0.1, 0.1, 0.1), 1.0), 4.0)
    g = orc.rhs_point(m.pts, m.nrm, [0.1, 0.1, 0.1], 1.0, 4.0)
    assert rel(f, g) < 1e-14


def test_solve_plain_fp64_uncorrected_vs_lu(bie, orc, cfg1):
    """cfg 1: corrections OFF vs O-dense (dense Dt + diag -> LU), sigma to 1e-12."""
    itf, m, Cm, A = cfg1
    b = orc.rhs_point(m.pts, m.nrm, [0.1, 0.1, 0.1], 1.0, 4.0)
    x_lu = sla.lu_solve(sla.lu_factor(A), b)
    assert np.linalg.norm(A @ x_lu - b) < 1e-10  # test/solver/dielectric_box3d.jl:10-18
    op = bie.lhs_dielectric_box3d(itf)
    x, st = bie.gpu_solve(op, b, rtol=1e-14, itmax=300)
    assert rel(x, x_lu) < 1e-12, (rel(x, x_lu), st)
    # total polarisation charge 1 - 1/eps (test/solver/dielectric_box3d.jl:26-30)
    assert abs(np.dot(m.w, x) + 1.0 / 4.0 - 1.0) < 1e-1


def test_solve_plain_fp64_corrected_vs_lu(bie, orc, cfg1):
    """cfg 1: corrections ON vs O-corr (dense Dt + C + diag -> LU)."""
    itf, m, Cm, A = cfg1
    b = orc.rhs_point(m.pts, m.nrm, [0.1, 0.1, 0.1], 1.0, 4.0)
    Ac = A + Cm.toarray()
    x_lu = sla.lu_solve(sla.lu_factor(Ac), b)
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    x, st = bie.gpu_solve(op, b, rtol=1e-14, itmax=300)
    assert rel(x, x_lu) < 1e-12, (rel(x, x_lu), st)
    x_or, it, _ = orc.gmres(m, b, Cm, atol=0.0, rtol=1e-13, itmax=300)
    assert rel(x_or, x_lu) < 1e-11


def test_solve_gmres_api(bie, orc, cfg1):
    itf, m, Cm, A = cfg1
    b = bie.rhs_dielectric_box3d(itf, bie.PointSource((0.1, 0.1, 0.1), 1.0), 4.0)
    op = bie.lhs_dielectric_box3d_fmm3d(itf, 1e-12)
    x = bie.solve_gmres(op, b, 1e-12, 1e-12)
    assert np.linalg.norm(A @ x - b) < 1e-10  # test/solver/dielectric_box3d.jl:23-24


@pytest.mark.parametrize("precision", ["fp32"])
def test_solve_refined_vs_lu(bie, orc, cfg1, precision):
    itf, m, Cm, A = cfg1
    Ac = A + Cm.toarray()
    src = np.array([[0.1, 0.1, 0.1], [-0.3, 0.2, 0.05], [0.2, -0.2, -0.1]])
    B = np.stack([orc.rhs_point(m.pts, m.nrm, s, q, 4.0) for s, q in zip(src, [1.0, -0.5, 2.0])], axis=1)
    X_lu = sla.lu_solve(sla.lu_factor(Ac), B)
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8, precision=precision)
    X, st = bie.gpu_solve(op, B, rtol=1e-11, itmax=400)
    assert st.solved and st.outer >= 1 and st.lowp_matvecs > 0
    for c in range(3):
        assert rel(X[:, c], X_lu[:, c]) < 1e-8


def test_block_equals_looped(bie, cfg1):
    """test/solver/multi_rhs.jl:59-66: block solve == looped single solves < 1e-6."""
    itf = cfg1[0]
    srcs = [bie.PointSource((0.1, 0.1, 0.1), 1.0), bie.PointSource((-0.2, 0.1, 0.0), -1.0)]
    S, st = bie.solve_dielectric_box3d_block(itf, srcs, 4.0, rtol=1e-10)
    op = bie.batched_lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-9, 1e-9, 8)
    for c, s in enumerate(srcs):
        f = bie.rhs_dielectric_box3d(itf, s, 4.0)
        x, _ = bie.gpu_solve(op, f, rtol=1e-10, precondition=True)
        assert np.max(np.abs(S[:, c] - x)) < 1e-6


def test_potential_and_energy(bie, orc, cfg1, rng):
    itf, m = cfg1[0], cfg1[1]
    S = rng.standard_normal((itf.n, 3))
    T = rng.uniform(-1, 1, (50, 3)) + np.array([2.0, 0, 0])
    phi = bie.laplace3d_pottrg(itf, T) @ S
    ref = orc.pottrg_apply(m.pts, m.w, T, S)
    assert rel(phi, ref) < 1e-13
    src = [bie.PointSource((0.1, 0.1, 0.1), 1.0), bie.PointSource((0.2, -0.1, 0.0), -2.0), bie.PointSource((0, 0, 0.1), 0.5)]
    W = bie.polarization_energy(itf, S, src)
    for c, s in enumerate(src):
        ref_c = 0.5 * s.charge * orc.pottrg_apply(m.pts, m.w, np.array([s.point]), S[:, c])[0]
        assert abs(W[c] - ref_c) <= 1e-13 * abs(ref_c)


@pytest.mark.parametrize("k", [16, 20, 64, 144])
def test_matvec_bf16x3_tensor_core(bie, cfg1, rng, k):
    """K3 (tcgen05 split-BF16 three-term contraction) vs the FP64 operator: the dropped
    lo*lo term and FP32 accumulation bound the error near 1e-5 relative."""
    itf = cfg1[0]
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-9, 1e-9, 8)
    X = rng.standard_normal((itf.n, k))
    Y64 = op.mul(X)
    Ytc = op.mul(X, precision="bf16x3")
    for c in range(k):
        assert rel(Ytc[:, c], Y64[:, c]) < 5e-5, (c, rel(Ytc[:, c], Y64[:, c]))
    # self-interaction excluded, corrections and diagonal intact: near the FP32 operator
    assert rel(Ytc, op.mul(X, precision="fp32")) < 5e-5


def test_solve_refined_bf16x3_vs_lu(bie, orc, cfg1, rng):
    itf, m, Cm, A = cfg1
    Ac = A + Cm.toarray()
    src = rng.uniform(-0.25, 0.25, (16, 3))
    q = rng.standard_normal(16)
    B = np.stack([orc.rhs_point(m.pts, m.nrm, s, qq, 4.0) for s, qq in zip(src, q)], axis=1)
    X_lu = sla.lu_solve(sla.lu_factor(Ac), B)
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8, precision="bf16x3")
    X, st = bie.gpu_solve(op, B, rtol=1e-11, itmax=400)
    assert st.solved and st.lowp_matvecs > 0
    for c in range(16):
        assert rel(X[:, c], X_lu[:, c]) < 1e-8


def test_matvec_bf16x6_tensor_core(bie, cfg1, rng):
    """Three bf16 pieces per operand, six products: FP32-level accuracy (residual updates)."""
    itf = cfg1[0]
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-9, 1e-9, 8)
    X = rng.standard_normal((itf.n, 32))
    Y64 = op.mul(X)
    Y6 = op.mul(X, precision="bf16x6")
    Y3 = op.mul(X, precision="bf16x3")
    assert rel(Y6, Y64) < 5e-7  # FP32-level: the FP32 kernel generation bounds it
    assert rel(Y6, Y64) < rel(Y3, Y64)


def test_tensor_core_accumulation_does_not_grow_with_n(bie, rng):
    """42048 nodes (657 source chunks per target tile): the FP32 tensor-memory sums are
    folded into a two-sum pair every 256 sources, so BF16x3 stays at the FP32-kernel
    level instead of growing with the number of sources."""
    itf = bie.single_dielectric_box3d(1.5, 1.0, 0.8, 6, 0.08, 4.0, 1.0)
    assert itf.n == 42048
    op = bie.lhs_dielectric_box3d(itf)
    X = rng.standard_normal((itf.n, 16))
    Y64 = op.mul(X)
    Y32 = op.mul(X, precision="fp32")
    Y3 = op.mul(X, precision="bf16x3")
    e32, e3 = rel(Y32, Y64), rel(Y3, Y64)
    assert e3 < 2e-6 and e3 < 3 * e32, (e3, e32)


@pytest.mark.parametrize("k", [1, 3, 8, 64, 128])
def test_combine_column_tiles(bie, cfg1, rng, k):
    """Block-row correction apply for every column-tile shape (k < 64, k = 64, k multiple of 64)."""
    itf, m, Cm, A = cfg1
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    X = rng.standard_normal((itf.n, k))
    Y = op @ X
    ref = A @ X + Cm @ X
    assert rel(Y, ref) < 1e-13


def test_autotuned_launch_recorded_and_accurate(bie, cfg1, rng):
    """The first tensor-core and FP64 applications tune their launch shape; results stay
    within the operators' bars (the split count only changes the partial-sum rounding)."""
    itf, m, Cm, A = cfg1
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    X = rng.standard_normal((itf.n, 24))
    Y64 = op.mul(X)
    Y3 = op.mul(X, precision="bf16x3")
    t_tc = bie.tuned_launch(op, "tensor_core", 24)
    t_64 = bie.tuned_launch(op, "fp64", 24)
    assert t_tc is not None and t_tc["nsplit"] >= 1 and t_tc["ctas_per_sm"] in (1, 2) and t_tc["ms"] > 0
    assert t_64 is not None and t_64["nsplit"] >= 1
    assert rel(Y64, A @ X + Cm @ X) < 1e-13
    assert rel(Y3, Y64) < 5e-5
    # widths of the same kernel instance share the entry: 17..32 columns run the 32-wide
    # tensor-core and FP64 instances tuned above, and reading them retunes nothing
    for kk in (17, 31, 32):
        assert bie.tuned_launch(op, "tensor_core", kk) == t_tc
        assert bie.tuned_launch(op, "fp64", kk) == t_64
    X2 = rng.standard_normal((itf.n, 19))
    assert rel(op.mul(X2, precision="bf16x3"), op.mul(X2)) < 5e-5
    assert bie.tuned_launch(op, "tensor_core", 19) == t_tc


def test_workspace_trim_keeps_results(bie, cfg1, monkeypatch):
    """Solves after the solver workspace was released (BIE_TRIM_WORKSPACE: after every
    solve) reallocate it and recapture their graphs, and give the same sigma."""
    itf, m, Cm, A = cfg1
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8, precision="bf16x3")
    src = [bie.PointSource((0.1, 0.1, 0.1), 1.0), bie.PointSource((-0.2, 0.05, 0.0), -0.5)] * 4
    F = bie.rhs_dielectric_box3d(itf, src, 4.0)
    S0, _ = bie.gpu_solve(op, F, rtol=1e-10)
    S1, _ = bie.gpu_solve(op, F, rtol=1e-10)
    monkeypatch.setenv("BIE_TRIM_WORKSPACE", "1")
    S2, st2 = bie.gpu_solve(op, F, rtol=1e-10)
    S3, st3 = bie.gpu_solve(op, F, rtol=1e-10)
    assert st2.solved and st3.solved
    for S in (S1, S2, S3):
        assert rel(S, S0) < 1e-13
