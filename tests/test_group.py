"""Several geometries in one launch: bie_matvec_group_device applies the split-BF16 operator
of three boxes of different node counts and column widths with ONE work-list launch of the
tensor-core direct sum over all their (target tile, source split) items
(mul!(Y, ::BatchedDielectricOperator, X), src/solver/multi_rhs.jl:103-136, for uneven
operators at once). With the launch shapes fixed by the model (BIE_NO_AUTOTUNE) it equals
each geometry's own launch to 1e-13 (the same arithmetic per tile); bie_solve_group_device
solves all three in lockstep and each sigma equals the geometry solved alone within the
refined bar (1e-8)."""
import ctypes as C

import numpy as np
import pytest

BOXES = [(1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0), (1.0, 0.6, 0.5, 6, 0.12, 10.0, 1.0), (0.8, 0.8, 0.8, 4, 0.25, 2.5, 1.0)]
KS = [24, 16, 40]


def test_group_entries_reject_bad_arguments(bie):
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    ks = (C.c_int32 * 1)(16)
    ptrs = (C.c_void_p * 1)(None)
    assert L.bie_matvec_group_device(None, 1, ptrs, ptrs, ks, _abi.BIE_BF16X3, 0, None) == _abi.BIE_EINVAL
    assert L.bie_solve_group_device(ptrs, 0, ptrs, ptrs, ks, None, None, None) == _abi.BIE_EINVAL


@pytest.fixture(scope="module")
def group(bie):
    import torch
    ops, X = [], []
    rng = np.random.default_rng(5)
    for b, k in zip(BOXES, KS):
        itf = bie.single_dielectric_box3d(*b)
        ops.append((itf, bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8), b))
        X.append(torch.from_numpy(rng.standard_normal((itf.n, k))).cuda())
    return ops, X


def ptr_array(ts):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


@pytest.mark.gpu
def test_group_matvec_equals_separate_launches(bie, group, monkeypatch):
    import torch
    from dielectricbie_jl_b200 import _abi
    monkeypatch.setenv("BIE_NO_AUTOTUNE", "1")
    L = _abi.lib()
    ops0, X = group
    # fresh geometries created with the autotuner off (the setting is read at creation)
    ops = [(itf, bie.GPUDielectricOperator(bie.single_dielectric_box3d(*b), precision="bf16x3"), b)
           for itf, _, b in ops0]
    assert len({itf.n for itf, _, _ in ops}) == 3
    Yg = [torch.empty_like(x) for x in X]
    Ys = [torch.empty_like(x) for x in X]
    gs = (C.c_void_p * 3)(*[op.geom._h.value for _, op, _ in ops])
    ks = (C.c_int32 * 3)(*KS)
    _abi.check(L.bie_matvec_group_device(gs, 3, ptr_array(X), ptr_array(Yg), ks, _abi.BIE_BF16X3, 0, None))
    for (itf, op, _), x, y, k in zip(ops, X, Ys, KS):
        _abi.check(L.bie_matvec_device(op.geom._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), k,
                                       _abi.BIE_BF16X3, 0, None))
    torch.cuda.synchronize()
    for a, b in zip(Yg, Ys):
        assert torch.isfinite(a).all()
        assert float((a - b).norm() / b.norm()) <= 1e-13


@pytest.mark.gpu
def test_group_solve_equals_alone(bie, group):
    import torch
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    ops, _ = group
    rng = np.random.default_rng(6)
    F = []
    for (itf, op, b), k in zip(ops, KS):
        half = 0.4 * np.array(b[:3])
        src = [bie.PointSource(tuple(rng.uniform(-half, half)), float(rng.standard_normal())) for _ in range(k)]
        F.append(torch.from_numpy(np.ascontiguousarray(bie.rhs_dielectric_box3d(itf, src, b[5]))).cuda())
    S = [torch.empty_like(f) for f in F]
    o = _abi.SolveOpts()
    L.bie_solve_opts_default(C.byref(o))
    o.rtol, o.precision = 1e-10, _abi.BIE_BF16X3
    st = (_abi.Stats * 3)()
    gs = (C.c_void_p * 3)(*[op.geom._h.value for _, op, _ in ops])
    ks = (C.c_int32 * 3)(*KS)
    _abi.check(L.bie_solve_group_device(gs, 3, ptr_array(F), ptr_array(S), ks, C.byref(o), st, None))
    torch.cuda.synchronize()
    for (itf, op, _), f, sg, t in zip(ops, F, S, st):
        assert t.converged and t.max_rel_resid <= 1e-10 * (1 + 1e-6)
        ref, rst = bie.gpu_solve(op, f.cpu().numpy(), rtol=1e-10, precision="bf16x3")
        got = sg.cpu().numpy()
        err = np.linalg.norm(got - ref, axis=0) / np.linalg.norm(ref, axis=0)
        assert err.max() < 1e-8, err.max()
