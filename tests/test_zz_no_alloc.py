"""bie_dt_apply_static: the direct sum that allocates no device memory.

Callers whose device memory is owned by a pool allocator (Julia's CUDA.jl,
PyTorch's caching allocator) or reserved at start-up by a latency-bound service
cannot let the library cudaMalloc its scratch; this entry point keeps its split
partials in a fixed 32 MiB array inside the library and takes every input and
output from the caller. Its output must match the regular entry point
(bie_matvec_device, FP64, no corrections, no diagonal) to the FP64 matvec
tolerance of the other parity tests, on consecutive calls that share the array.

The file name makes pytest collect it last; the GPU test passes alone in a fresh
process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)
RTOL = 1e-13  # FP64 matvec tolerance of the parity tests


def _static_call(L, cols, n, X_ptr, k, Y_ptr):
    return L.bie_dt_apply_static(*cols, n, X_ptr, k, Y_ptr, None)


def test_static_entry_rejects_bad_sizes_before_device_work(bie):
    """Sizes above the scratch limit and null pointers are refused on the host,
    with a message, before any CUDA call (so this runs without a GPU)."""
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    buf = np.zeros(8)
    p = C.c_void_p(buf.ctypes.data)
    cols = [p] * 7
    rc = _static_call(L, cols, (1 << 22) + 1, p, 1, p)
    assert rc == _abi.BIE_EINVAL
    msg = _abi.last_error()
    assert "exceeds the maximum of 4194304" in msg and "32 MiB" in msg
    rc = _static_call(L, [p] * 6 + [None], 16, p, 1, p)
    assert rc == _abi.BIE_EINVAL and "bad argument" in _abi.last_error()
    rc = _static_call(L, cols, 16, p, 0, p)
    assert rc == _abi.BIE_EINVAL


# the small box, and a 94,752-node box on which the scratch bound limits the column group
# (4,194,304 / n = 44 < 64 columns, so 70 columns run as 44 + 26) and the source splits (1)
BOXES = [CFG1, (2.0, 1.0, 1.0, 6, 0.05, 10.0, 1.0)]


@pytest.mark.gpu
@pytest.mark.parametrize("box", BOXES)
def test_static_entry_matches_matvec_device_on_consecutive_calls(bie, box):
    import torch
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    itf = bie.single_dielectric_box3d(*box)
    n = itf.n
    op = bie.lhs_dielectric_box3d(itf)  # regular path: geometry handle with its own buffers
    g = op.geom._h

    def d(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)

    pts, nrm = d(itf.points), d(itf.normals)
    cols_t = [pts[:, 0].contiguous(), pts[:, 1].contiguous(), pts[:, 2].contiguous(),
              nrm[:, 0].contiguous(), nrm[:, 1].contiguous(), nrm[:, 2].contiguous(), d(itf.weights)]
    cols = [C.c_void_p(t.data_ptr()) for t in cols_t]
    rng = np.random.default_rng(77)
    flags = _abi.BIE_NO_CORRECTIONS | _abi.BIE_NO_DIAG
    # 70 columns (two column groups), then 3: the second call finds the first one's
    # partials in the shared array
    for k in (70, 3):
        X = d(rng.standard_normal((n, k)))  # node-major n x k
        Y_static = torch.full((n, k), float("nan"), dtype=torch.float64, device=dev)
        Y_ref = torch.empty((n, k), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        _abi.check(_static_call(L, cols, n, C.c_void_p(X.data_ptr()), k, C.c_void_p(Y_static.data_ptr())))
        _abi.check(L.bie_matvec_device(g, C.c_void_p(X.data_ptr()), C.c_void_p(Y_ref.data_ptr()), k,
                                       _abi.BIE_FP64, flags, None))
        torch.cuda.synchronize()
        # a repeated call allocates nothing: the device's free memory is unchanged
        free0 = torch.cuda.mem_get_info(dev)[0]
        _abi.check(_static_call(L, cols, n, C.c_void_p(X.data_ptr()), k, C.c_void_p(Y_static.data_ptr())))
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info(dev)[0] == free0
        a, b = Y_static.cpu().numpy(), Y_ref.cpu().numpy()
        assert np.isfinite(a).all()
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < RTOL, (k, err)
        for c in range(k):
            assert np.linalg.norm(a[:, c] - b[:, c]) <= RTOL * np.linalg.norm(b[:, c]), (k, c)
