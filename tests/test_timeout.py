"""Failure detection without a GPU fault: the tensor-core kernel's mbarrier waits are
bounded. With BIE_TEST_TC_STALL set, every CTA's first right-hand-side tile is announced
but never copied, so the waits run out (a short limit in this mode), the CTAs release
their tensor memory and return, and the call reports BIE_ETIMEOUT; the handle and the
CUDA context stay usable afterwards."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def test_tensor_core_wait_timeout_is_reported_and_recoverable(bie):
    from dielectricbie_jl_b200 import _abi
    itf = bie.single_dielectric_box3d(*CFG1)
    op = bie.lhs_dielectric_box3d(itf)
    X = np.random.default_rng(5).standard_normal((itf.n, 16))
    Y64 = op.mul(X)
    Y_ok = op.mul(X, precision="bf16x3")  # tunes the launch before the stalled call
    os.environ["BIE_TEST_TC_STALL"] = "1"
    try:
        with pytest.raises(_abi.BieError) as e:
            op.mul(X, precision="bf16x3")
        assert e.value.code == _abi.BIE_ETIMEOUT
        assert "wait" in str(e.value)
    finally:
        del os.environ["BIE_TEST_TC_STALL"]
    Y = op.mul(X, precision="bf16x3")
    assert np.linalg.norm(Y - Y64) / np.linalg.norm(Y64) < 5e-5
    assert np.array_equal(Y, Y_ok) or np.linalg.norm(Y - Y_ok) / np.linalg.norm(Y_ok) < 1e-12
    assert np.linalg.norm(op.mul(X) - Y64) == 0.0
