"""Streaming correction apply (K4 for k <= 16 on meshes with many block rows, the
bulk-copy pipeline of combine_bulk.cu) on the cfg3 box, N = 42,048, n_quad = 6.

It agrees with the block-row kernel (BIE_COMBINE_ROWS forces that form) to 1e-14: the
block-row form splits the long rows of this mesh into groups summed separately, so the
two round differently. The operator matches the oracle's matrix-free corrected operator
(direct sum + CSC corrections + diagonal, src/kernel/laplace3d_near.jl:395-419) to 1e-13."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG3 = (1.5, 1.0, 0.8, 6, 0.08, 4.0, 1.0)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope="module")
def cfg3(bie):
    # eager launches (no CUDA graphs) on this handle, so each solve takes the combine
    # form selected at the time of the call
    itf = bie.single_dielectric_box3d(*CFG3)
    os.environ["BIE_NO_GRAPHS"] = "1"
    try:
        op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    finally:
        del os.environ["BIE_NO_GRAPHS"]
    return itf, op


def rows_form(fn):
    os.environ["BIE_COMBINE_ROWS"] = "1"
    try:
        return fn()
    finally:
        del os.environ["BIE_COMBINE_ROWS"]


@pytest.mark.parametrize("k", [1, 2, 3, 8, 12, 16])
def test_streaming_equals_block_rows_fp64(cfg3, rng, k):
    itf, op = cfg3
    X = rng.standard_normal((itf.n, k))
    Y = op.mul(X)
    Yr = rows_form(lambda: op.mul(X))
    assert rel(Y, Yr) < 1e-14


@pytest.mark.parametrize("precision,k", [("fp32", 2), ("bf16x3", 8), ("bf16x3", 16)])
def test_streaming_equals_block_rows_low_precision(cfg3, rng, precision, k):
    """FP32 split partials of the tensor-core sum (bf16x3) and FP64 partials (fp32)."""
    itf, op = cfg3
    X = rng.standard_normal((itf.n, k))
    Y = op.mul(X, precision=precision)
    Yr = rows_form(lambda: op.mul(X, precision=precision))
    assert rel(Y, Yr) < 1e-14


def test_streaming_matches_oracle(bie, orc, cfg3):
    itf, op = cfg3
    m = orc.Mesh.single_box(*CFG3)
    assert m.n == itf.n
    ups, adp = orc.build_neighbor_list(m, 8, 1e-9, True)
    Cm = orc.DT_corrections(m, ups, adp, 1e-9)
    j = np.arange(1, itf.n + 1)
    X = np.stack([np.cos(0.2 * j), np.sin(0.013 * j) + 0.5], axis=1)
    Y = op.mul(X)
    for c in range(2):
        assert rel(Y[:, c], orc.op_apply(m, X[:, c], Cm)) < 1e-13


def test_streaming_with_preconditioner_in_solve(bie, cfg3):
    """The preconditioned slab (p .* X) is streamed too: a right-preconditioned refined
    solve gives the same sigma through either form (to the solve's own accuracy)."""
    itf, op = cfg3
    rng = np.random.default_rng(31)
    F = np.stack([bie.rhs_dielectric_box3d(itf, bie.PointSource(tuple(rng.uniform(-0.3, 0.3, 3)),
                                                                   float(rng.standard_normal())), 4.0)
                  for _ in range(8)], axis=1)
    S, st = bie.gpu_solve(op, F, rtol=1e-10, precision="bf16x3", precondition=True)
    Sr, str_ = rows_form(lambda: bie.gpu_solve(op, F, rtol=1e-10, precision="bf16x3", precondition=True))
    assert st.solved and str_.solved
    assert rel(S, Sr) < 1e-9
