"""bie_solve_point (point-source right-hand sides built on the device and solved in one
call, rhs_dielectric_box3d + solve_dielectric_box3d_block, src/solver/dielectric_box3d.jl:95-104
and src/solver/multi_rhs.jl:270-286) equals bie_rhs_point followed by bie_solve on the same
geometry bit for bit, and rejects bad arguments before touching the device."""
import ctypes as C

import numpy as np
import pytest

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def test_solve_point_rejects_bad_arguments(bie):
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    src = np.zeros((1, 3))
    q = np.ones(1)
    S = np.zeros(4)
    assert L.bie_solve_point(None, _abi.dptr(src), _abi.dptr(q), _abi.dptr(q), 1, _abi.dptr(S), None,
                             None) == _abi.BIE_EINVAL
    assert "solve_point" in _abi.last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("k,precision", [(1, "fp64"), (8, "fp64"), (20, "bf16x3")])
def test_solve_point_equals_rhs_then_solve(bie, k, precision):
    itf = bie.single_dielectric_box3d(*CFG1)
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    rng = np.random.default_rng(k)
    srcs = [bie.PointSource(tuple(rng.uniform(-0.25, 0.25, 3)), float(rng.standard_normal())) for _ in range(k)]
    F = bie.rhs_dielectric_box3d(itf, srcs, 4.0)
    S1, st1 = bie.gpu_solve(op, F.reshape(itf.n, k), rtol=1e-11, precision=precision)
    S2, st2 = bie.gpu_solve_sources(op, srcs, 4.0, rtol=1e-11, precision=precision)
    assert st1.solved and st2.solved and st1.iterations == st2.iterations
    assert np.array_equal(S1, S2)
    # the block API (block GMRES by default, as Krylov.block_gmres) is the same call
    S3, _ = bie.solve_dielectric_box3d_block(itf, srcs, 4.0, rtol=1e-11, precision=precision, precondition=False)
    S4, _ = bie.gpu_solve_sources(op, srcs, 4.0, rtol=1e-11, precision=precision, block=True)
    assert np.array_equal(S3, S4)
    S5, _ = bie.solve_dielectric_box3d_block(itf, srcs, 4.0, rtol=1e-11, precision=precision, precondition=False,
                                             block=False)
    assert np.array_equal(S5, S2)
