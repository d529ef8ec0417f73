"""ctypes binding of libbie_b200.so (the C ABI declared in include/bie_b200.h).

Only plain pointers and sizes cross the boundary. The library is required: if it
is missing this module raises on first use (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbie_b200.so")

BIE_OK, BIE_EINVAL, BIE_ENOMEM, BIE_ECUDA, BIE_ENOCONV, BIE_ETIMEOUT, BIE_EUNSUPPORTED, BIE_ENODEVICE = range(8)
BIE_FP64, BIE_FP32, BIE_BF16X3, BIE_BF16X6 = 0, 1, 2, 3
BIE_NO_CORRECTIONS, BIE_NO_DIAG, BIE_NO_VERIFY = 1, 2, 4
PRECISIONS = {"fp64": BIE_FP64, "fp32": BIE_FP32, "bf16x3": BIE_BF16X3, "bf16x6": BIE_BF16X6}

# Every symbol the header declares (checked by the CPU test suite).
EXPORTS = [
    "bie_last_error", "bie_version", "bie_device_count", "bie_gausslegendre", "bie_best_grid",
    "bie_mesh_single_box", "bie_mesh_multi_box", "bie_mesh_from_panels", "bie_mesh_info", "bie_mesh_copy",
    "bie_mesh_destroy", "bie_near_opts_default", "bie_near_build", "bie_near_info", "bie_near_copy",
    "bie_near_release_values", "bie_near_destroy", "bie_geom_near_values", "bie_geom_create", "bie_geom_create_from_mesh", "bie_geom_info", "bie_geom_stream",
    "bie_geom_destroy", "bie_matvec", "bie_matvec_device", "bie_rhs_point", "bie_rhs_point_device",
    "bie_potential", "bie_potential_device", "bie_energy", "bie_solve_opts_default", "bie_solve", "bie_solve_point",
    "bie_matvec_group_device", "bie_solve_group_device",
    "bie_solve_device", "bie_profile_enable", "bie_profile_read", "bie_dt_apply_static",
    "bie_server_opts_default", "bie_server_create", "bie_server_submit", "bie_server_submit_point",
    "bie_server_poll",
    "bie_server_counters_read", "bie_server_destroy", "bie_tuning_read", "bie_peak_probe",
    "bie_probe_create", "bie_probe_info", "bie_probe_copy", "bie_probe_apply", "bie_probe_destroy",
]


class BieError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libbie_b200 error {code}: {msg}")
        self.code = code


class NotConverged(BieError):
    pass


class NearOpts(C.Structure):
    _fields_ = [("max_order", C.c_int), ("up_tol", C.c_double), ("correct_edges", C.c_int),
                ("adaptive_atol", C.c_double), ("adaptive_rtol", C.c_double), ("adaptive_n_GL", C.c_int),
                ("adaptive_max_depth", C.c_int), ("nthreads", C.c_int), ("device", C.c_int)]


class SolveOpts(C.Structure):
    _fields_ = [("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_int), ("restart", C.c_int),
                ("precision", C.c_int), ("inner_rtol", C.c_double), ("max_outer", C.c_int),
                ("precondition", C.c_int), ("check_every", C.c_int), ("flags", C.c_uint32), ("block", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("max_slots", C.c_int), ("max_batch_rhs", C.c_int), ("hbm_fraction", C.c_double),
                ("device", C.c_int), ("max_group", C.c_int)]


class ServerCounters(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("batches", C.c_int64),
                ("merged_requests", C.c_int64), ("queued", C.c_int64), ("inflight", C.c_int),
                ("peak_inflight", C.c_int), ("hbm_budget", C.c_int64), ("hbm_in_use", C.c_int64),
                ("hbm_peak", C.c_int64), ("workspace_releases", C.c_int64), ("enomem_retries", C.c_int64),
                ("groups", C.c_int64), ("grouped_batches", C.c_int64)]


class KernelTime(C.Structure):
    _fields_ = [("ms", C.c_double), ("launches", C.c_int64), ("pairs", C.c_double), ("pair_cols", C.c_double),
                ("bytes", C.c_double)]


KERNEL_KINDS = {"direct_fp64": 0, "direct_fp32": 1, "direct_tc": 2, "combine": 3, "krylov": 4, "other": 5, "all": 6}


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer", C.c_int), ("fp64_matvecs", C.c_int), ("lowp_matvecs", C.c_int),
                ("converged", C.c_int), ("max_rel_resid", C.c_double), ("seconds", C.c_double),
                ("col_iterations", C.POINTER(C.c_int)), ("col_resid", C.POINTER(C.c_double))]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i32p = C.POINTER(C.c_int32)
_vp = C.c_void_p
_lib = None


def lib():
    """Load libbie_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python dielectricbie.jl_b200/build.py`")
    L = C.CDLL(LIB_PATH)
    i, d, i64, u32 = C.c_int, C.c_double, C.c_int64, C.c_uint32
    sig = {
        "bie_last_error": (i, [C.c_char_p, C.c_size_t]),
        "bie_version": (C.c_char_p, []),
        "bie_device_count": (i, []),
        "bie_gausslegendre": (i, [i, _dp, _dp]),
        "bie_best_grid": (i, [d, d, d, _ip, _ip]),
        "bie_mesh_single_box": (i, [d, d, d, i, d, d, d, d, C.POINTER(_vp)]),
        "bie_mesh_multi_box": (i, [i, d, i, _dp, _dp, _dp, d, d, C.POINTER(_vp)]),
        "bie_mesh_from_panels": (i, [i, i, _dp, _dp, _ip, _dp, _dp, C.POINTER(_vp)]),
        "bie_mesh_info": (i, [_vp, C.POINTER(i64), _ip, _ip]),
        "bie_mesh_copy": (i, [_vp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp, _dp]),
        "bie_mesh_destroy": (None, [_vp]),
        "bie_near_opts_default": (None, [C.POINTER(NearOpts)]),
        "bie_near_build": (i, [_vp, C.POINTER(NearOpts), C.POINTER(_vp)]),
        "bie_near_info": (i, [_vp, C.POINTER(i64), _ip, _ip, _ip, _ip]),
        "bie_near_copy": (i, [_vp, _i32p, _i32p, _dp, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "bie_near_destroy": (None, [_vp]),
        "bie_near_release_values": (i, [_vp]),
        "bie_geom_near_values": (i, [_vp, _dp, i64]),
        "bie_geom_create": (i, [_dp, _dp, _dp, _dp, i64, C.c_int32, C.c_int32, _i32p, _i32p, _dp, i64, i,
                                C.POINTER(_vp)]),
        "bie_geom_create_from_mesh": (i, [_vp, _vp, i, C.POINTER(_vp)]),
        "bie_geom_info": (i, [_vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_size_t)]),
        "bie_geom_stream": (_vp, [_vp]),
        "bie_geom_destroy": (None, [_vp]),
        "bie_matvec": (i, [_vp, _dp, _dp, C.c_int32, C.c_int32, u32]),
        "bie_matvec_device": (i, [_vp, _vp, _vp, C.c_int32, C.c_int32, u32, _vp]),
        "bie_rhs_point": (i, [_vp, _dp, _dp, _dp, C.c_int32, _dp]),
        "bie_rhs_point_device": (i, [_vp, _vp, _vp, _vp, C.c_int32, _vp, _vp]),
        "bie_potential": (i, [_vp, _dp, C.c_int32, _dp, i64, _dp]),
        "bie_potential_device": (i, [_vp, _vp, C.c_int32, _vp, i64, _vp, _vp]),
        "bie_energy": (i, [_vp, _dp, C.c_int32, _dp, _dp, _dp]),
        "bie_probe_create": (i, [_vp, _dp, C.c_int64, C.c_double, C.c_double, C.c_int32, C.POINTER(_vp)]),
        "bie_probe_info": (i, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                               C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "bie_probe_copy": (i, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _dp, _dp, _dp,
                               C.POINTER(C.c_int64), C.POINTER(C.c_int32), _dp,
                               C.POINTER(C.c_int64), C.POINTER(C.c_int32), _dp]),
        "bie_probe_apply": (i, [_vp, _dp, C.c_int32, _dp]),
        "bie_probe_destroy": (None, [_vp]),
        "bie_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
        "bie_solve": (i, [_vp, _dp, _dp, C.c_int32, C.POINTER(SolveOpts), C.POINTER(Stats)]),
        "bie_solve_point": (i, [_vp, _dp, _dp, _dp, C.c_int32, _dp, C.POINTER(SolveOpts), C.POINTER(Stats)]),
        "bie_matvec_group_device": (i, [C.POINTER(_vp), C.c_int32, C.POINTER(_vp), C.POINTER(_vp),
                                        C.POINTER(C.c_int32), C.c_int32, C.c_uint32, _vp]),
        "bie_solve_group_device": (i, [C.POINTER(_vp), C.c_int32, C.POINTER(_vp), C.POINTER(_vp),
                                       C.POINTER(C.c_int32), C.POINTER(SolveOpts), C.POINTER(Stats), _vp]),
        "bie_solve_device": (i, [_vp, _vp, _vp, C.c_int32, C.POINTER(SolveOpts), C.POINTER(Stats), _vp]),
        "bie_profile_enable": (i, [_vp, i]),
        "bie_profile_read": (i, [_vp, i, C.POINTER(KernelTime)]),
        "bie_dt_apply_static": (i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, i64, _vp, C.c_int32, _vp, _vp]),
        "bie_server_opts_default": (None, [C.POINTER(ServerOpts)]),
        "bie_server_create": (i, [C.POINTER(ServerOpts), C.POINTER(_vp)]),
        "bie_server_submit": (i, [_vp, _vp, _dp, C.c_int32, C.POINTER(SolveOpts), C.POINTER(C.c_uint64)]),
        "bie_server_submit_point": (i, [_vp, _vp, _dp, _dp, _dp, C.c_int32, C.POINTER(SolveOpts), C.POINTER(C.c_uint64)]),
        "bie_server_poll": (i, [_vp, C.c_uint64, C.c_int32, _dp, C.POINTER(Stats), C.POINTER(C.c_double),
                                C.POINTER(C.c_int)]),
        "bie_server_counters_read": (i, [_vp, C.POINTER(ServerCounters)]),
        "bie_server_destroy": (None, [_vp]),
        "bie_tuning_read": (i, [_vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_double)]),
        "bie_peak_probe": (i, [C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib().bie_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc == BIE_OK:
        return
    msg = last_error()
    if rc == BIE_ENOCONV:
        raise NotConverged(rc, msg or "solver did not converge")
    raise BieError(rc, msg)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype in (np.int32, np.intc)
    return a.ctypes.data_as(_ip)


def i32ptr(a: np.ndarray):
    assert a.dtype == np.int32
    return a.ctypes.data_as(_i32p)


def device_count() -> int:
    return int(lib().bie_device_count())


def version() -> str:
    return lib().bie_version().decode()
