"""ctypes wrapper of the CPU oracle (``oracle/bie_oracle.c``).

Test infrastructure only: the parity checker for the CUDA library and the timed
CPU baseline leg of ``bench.py``. The product never imports this module.

Each wrapper names the reference function it restates (DielectricBIE.jl paths).
Layouts follow the reference's Julia SoA gather (``src/kernel/laplace3d.jl:85-97``):
points/normals are ``(N, 3)`` C-contiguous (== 3 x N column-major), multi-column
vectors are ``(N, k)`` Fortran-ordered (== Julia's N x k).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libbie_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_int64)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (into oracle/_build/)."""
    src = os.path.join(_HERE, "bie_oracle.c")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_SO)
        L.orc_gausslegendre.argtypes = [C.c_int, _dp, _dp]
        L.orc_best_grid.argtypes = [C.c_double, C.c_double, C.c_double, _ip, _ip]
        L.orc_best_grid.restype = C.c_int
        L.orc_mesh_single_box.argtypes = [C.c_double] * 3 + [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_mesh_single_box.restype = C.c_void_p
        L.orc_mesh_multi_box.argtypes = [C.c_int, C.c_double, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double]
        L.orc_mesh_multi_box.restype = C.c_void_p
        L.orc_mesh_from_panels.argtypes = [C.c_int, C.c_int, _dp, _dp, _ip, _dp, _dp]
        L.orc_mesh_from_panels.restype = C.c_void_p
        L.orc_mesh_free.argtypes = [C.c_void_p]
        L.orc_mesh_npanels.argtypes = [C.c_void_p]
        L.orc_mesh_nq.argtypes = [C.c_void_p]
        L.orc_mesh_npoints.argtypes = [C.c_void_p]
        L.orc_mesh_npoints.restype = C.c_int64
        L.orc_mesh_copy.argtypes = [C.c_void_p, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp]
        L.orc_pot.argtypes = [_dp, _dp]
        L.orc_pot.restype = C.c_double
        L.orc_grad.argtypes = [_dp, _dp, _dp]
        L.orc_grad.restype = C.c_double
        L.orc_diag.argtypes = [C.c_void_p, _dp]
        L.orc_DT_dense.argtypes = [C.c_void_p, _dp, C.c_int]
        L.orc_S_dense.argtypes = [C.c_void_p, _dp]
        L.orc_DT_apply.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.orc_pottrg_apply.argtypes = [C.c_int64, _dp, _dp, C.c_int64, _dp, _dp, _dp, C.c_int, C.c_int]
        L.orc_rhs_point.argtypes = [C.c_int64, _dp, _dp, _dp, C.c_double, C.c_double, _dp]
        L.orc_bernstein_rho_panel.argtypes = [_dp, _dp, _dp]
        L.orc_bernstein_rho_panel.restype = C.c_double
        L.orc_build_neighbor_list.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
        L.orc_build_neighbor_list.restype = C.c_void_p
        L.orc_nbr_free.argtypes = [C.c_void_p]
        L.orc_nbr_counts.argtypes = [C.c_void_p, _ip, _ip]
        L.orc_nbr_copy.argtypes = [C.c_void_p, _ip, _ip, _ip, _ip, _ip]
        L.orc_DT_panel.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.orc_DT_panel_upsampled.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_DT_panel_adaptive.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                            _dp, _ip]
        L.orc_DT_panel_adaptive.restype = C.c_int
        L.orc_adaptive_panel_moments.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int,
                                                 C.c_int, _dp]
        L.orc_adaptive_panel_moments.restype = C.c_int
        L.orc_DT_corrections.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
        L.orc_DT_corrections.restype = C.c_void_p
        L.orc_coo_free.argtypes = [C.c_void_p]
        L.orc_coo_nnz.argtypes = [C.c_void_p]
        L.orc_coo_nnz.restype = C.c_int64
        L.orc_coo_hit_max.argtypes = [C.c_void_p]
        L.orc_coo_copy.argtypes = [C.c_void_p, _lp, _lp, _dp]
        L.orc_op_apply.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _lp, _lp, _dp, _dp, _dp, C.c_int]
        L.orc_gmres.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _lp, _lp, _dp, _dp, _dp, C.c_double, C.c_double,
                                C.c_int, C.c_int, _dp]
        L.orc_gmres.restype = C.c_int
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _l(a):
    return a.ctypes.data_as(_lp) if a is not None else None


def _cd(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def gausslegendre(n: int):
    """FastGaussQuadrature.jl 1.1.0 ``gausslegendre`` (nodes ascending)."""
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gausslegendre(n, _d(x), _d(w))
    return x, w


def best_grid_mn(W, H, alpha):
    """``best_grid_mn`` (src/utils/best_grid.jl:8-126)."""
    m = C.c_int(0)
    n = C.c_int(0)
    rc = lib().orc_best_grid(float(W), float(H), float(alpha), C.byref(m), C.byref(n))
    if rc == -1:
        raise ValueError("W and H must be positive and alpha >= 1")
    if rc != 0:
        raise ValueError("no (m, n) found within search limits")
    return m.value, n.value


class Mesh:
    """A ``DielectricInterface`` of flat panels (src/core/panels.jl:5-118)."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("oracle mesher failed")
        self.h = C.c_void_p(handle)
        L = lib()
        self.npanels = L.orc_mesh_npanels(self.h)
        self.nq = L.orc_mesh_nq(self.h)
        self.n = int(L.orc_mesh_npoints(self.h))
        P, N = self.npanels, self.n
        self.corners = np.zeros((P, 4, 3))
        self.normals = np.zeros((P, 3))
        self.is_edge = np.zeros(P, dtype=np.int32)
        self.eps_in = np.zeros(P)
        self.eps_out = np.zeros(P)
        self.pts = np.zeros((N, 3))
        self.nrm = np.zeros((N, 3))
        self.w = np.zeros(N)
        L.orc_mesh_copy(self.h, _d(self.corners), _d(self.normals), _i(self.is_edge), _d(self.eps_in),
                        _d(self.eps_out), _d(self.pts), _d(self.nrm), _d(self.w))

    def __del__(self):
        try:
            lib().orc_mesh_free(self.h)
        except Exception:
            pass

    @classmethod
    def single_box(cls, Lx, Ly, Lz, nq, l_ec, eps_in, eps_out, alpha=np.sqrt(2.0)):
        """``single_dielectric_box3d`` (src/shape/box3d_single.jl:49-70)."""
        return cls(lib().orc_mesh_single_box(Lx, Ly, Lz, nq, l_ec, eps_in, eps_out, alpha))

    @classmethod
    def multi_box(cls, nq, l_ec, centers, dims, epses, eps_out=1.0, alpha=np.sqrt(2.0)):
        """``multi_dielectric_box3d`` (src/shape/box3d_multi.jl:358-386)."""
        c = _cd(centers, (-1, 3))
        d = _cd(dims, (-1, 3))
        e = _cd(epses)
        return cls(lib().orc_mesh_multi_box(nq, l_ec, len(e), _d(c), _d(d), _d(e), eps_out, alpha))

    @classmethod
    def from_panels(cls, nq, corners, normals, is_edge=None, eps_in=None, eps_out=None):
        """Interface from explicit ``rect_panel3d_discretize`` panels (src/shape/box3d.jl:22-64)."""
        c = _cd(corners, (-1, 4, 3))
        P = c.shape[0]
        n = _cd(normals, (P, 3))
        ie = np.ascontiguousarray(np.zeros(P) if is_edge is None else is_edge, dtype=np.int32)
        ei = _cd(np.full(P, 2.0) if eps_in is None else eps_in)
        eo = _cd(np.full(P, 1.0) if eps_out is None else eps_out)
        return cls(lib().orc_mesh_from_panels(P, nq, _d(c), _d(n), _i(ie), _d(ei), _d(eo)))

    def diag(self):
        """Per-node t_P = (eps_out+eps_in)/(2(eps_out-eps_in)) (src/solver/dielectric_box3d.jl:5-15)."""
        out = np.zeros(self.n)
        lib().orc_diag(self.h, _d(out))
        return out

    def DT_dense(self, with_diag=False):
        """``laplace3d_DT`` (+ ``lhs_dielectric_box3d`` with the diagonal)."""
        A = np.zeros((self.n, self.n), order="F")
        lib().orc_DT_dense(self.h, _d(A), int(with_diag))
        return A

    def S_dense(self):
        """``laplace3d_S`` (src/kernel/laplace3d.jl:18-28)."""
        A = np.zeros((self.n, self.n), order="F")
        lib().orc_S_dense(self.h, _d(A))
        return A


def pot(src, trg):
    return lib().orc_pot(_d(_cd(src)), _d(_cd(trg)))


def grad(src, trg, n):
    """``laplace3d_grad`` (src/kernel/laplace3d.jl:9-15)."""
    return lib().orc_grad(_d(_cd(src)), _d(_cd(trg)), _d(_cd(n)))


def DT_apply(pts, nrm, w, X, nthreads=0):
    """Direct D^T sum, j != i (the exact sum that lfmm3d pg=2 approximates)."""
    X = np.asarray(X, dtype=np.float64)
    vec = X.ndim == 1
    Xf = np.asfortranarray(X.reshape(X.shape[0], -1))
    N, k = Xf.shape
    Y = np.zeros((N, k), order="F")
    lib().orc_DT_apply(N, _d(_cd(pts)), _d(_cd(nrm)), _d(_cd(w)), _d(Xf), _d(Y), k, nthreads)
    return Y[:, 0] if vec else Y


def pottrg_apply(pts, w, targets, X, nthreads=0):
    """S[X](targets) (``laplace3d_pottrg`` action, src/kernel/laplace3d.jl:69-82)."""
    X = np.asarray(X, dtype=np.float64)
    vec = X.ndim == 1
    Xf = np.asfortranarray(X.reshape(X.shape[0], -1))
    N, k = Xf.shape
    T = _cd(targets, (-1, 3))
    M = T.shape[0]
    Y = np.zeros((M, k), order="F")
    lib().orc_pottrg_apply(N, _d(_cd(pts)), _d(_cd(w)), M, _d(T), _d(Xf), _d(Y), k, nthreads)
    return Y[:, 0] if vec else Y


def rhs_point(pts, nrm, src, q, eps_src):
    """``rhs_dielectric_box3d(::PointSource)`` (src/solver/dielectric_box3d.jl:95-104)."""
    pts = _cd(pts)
    out = np.zeros(pts.shape[0])
    lib().orc_rhs_point(pts.shape[0], _d(pts), _d(_cd(nrm)), _d(_cd(src)), float(q), float(eps_src), _d(out))
    return out


def bernstein_rho_panel(corners, normal, trg):
    """``bernstein_rho_panel`` (src/utils/bernstein.jl:33-62)."""
    return lib().orc_bernstein_rho_panel(_d(_cd(corners)), _d(_cd(normal)), _d(_cd(trg)))


def build_neighbor_list(mesh: Mesh, max_order: int, atol: float, correct_edges: bool = False):
    """``build_neighbor_list`` (src/kernel/laplace3d_near.jl:240-392), 0-based panel ids.

    Returns (upsample: dict (i, j) -> p_up, adaptive: list of (i, j))."""
    L = lib()
    h = L.orc_build_neighbor_list(mesh.h, max_order, atol, int(bool(correct_edges)))
    nu, na = C.c_int(0), C.c_int(0)
    L.orc_nbr_counts(h, C.byref(nu), C.byref(na))
    ui = np.zeros(nu.value, dtype=np.int32)
    uj = np.zeros(nu.value, dtype=np.int32)
    up = np.zeros(nu.value, dtype=np.int32)
    ai = np.zeros(na.value, dtype=np.int32)
    aj = np.zeros(na.value, dtype=np.int32)
    L.orc_nbr_copy(h, _i(ui), _i(uj), _i(up), _i(ai), _i(aj))
    L.orc_nbr_free(h)
    ups = {(int(i), int(j)): int(p) for i, j, p in zip(ui, uj, up)}
    adp = [(int(i), int(j)) for i, j in zip(ai, aj)]
    return ups, adp


def _nbr_handle(mesh, ups, adp):
    """Rebuild a C neighbour list from python dict/list (for corrections)."""
    class _N(C.Structure):
        _fields_ = [("n_ups", C.c_int), ("n_adp", C.c_int), ("ups_i", _ip), ("ups_j", _ip), ("ups_p", _ip),
                    ("adp_i", _ip), ("adp_j", _ip)]
    keys = sorted(ups)
    ui = np.array([k[0] for k in keys], dtype=np.int32)
    uj = np.array([k[1] for k in keys], dtype=np.int32)
    up = np.array([ups[k] for k in keys], dtype=np.int32)
    a = sorted(adp)
    ai = np.array([k[0] for k in a], dtype=np.int32)
    aj = np.array([k[1] for k in a], dtype=np.int32)
    s = _N(len(keys), len(a), _i(ui), _i(uj), _i(up), _i(ai), _i(aj))
    return s, (ui, uj, up, ai, aj)


def DT_panel(mesh, src, trg):
    """``laplace3d_DT_panel`` (src/kernel/laplace3d_near.jl:25-34), (np_trg, np_src)."""
    nq2 = mesh.nq ** 2
    out = np.zeros((nq2, nq2))
    lib().orc_DT_panel(mesh.h, src, trg, _d(out))
    return out


def DT_panel_upsampled(mesh, src, trg, n_up):
    """``laplace3d_DT_panel_upsampled`` (src/kernel/laplace3d_near_upsampling.jl:52-119)."""
    nq2 = mesh.nq ** 2
    out = np.zeros((nq2, nq2))
    lib().orc_DT_panel_upsampled(mesh.h, src, trg, n_up, _d(out))
    return out


def DT_panel_adaptive(mesh, src, trg, atol, rtol=np.sqrt(np.finfo(float).eps), n_GL=0, max_depth=20):
    """Touching-pair block (walk_adaptive_tree + adaptive_block_moments_inplace!,
    src/kernel/laplace3d_near_adaptive.jl:119-224, 308-387). Returns (block, hit_max, n_leaves)."""
    nq2 = mesh.nq ** 2
    out = np.zeros((nq2, nq2))
    nl = C.c_int(0)
    hm = lib().orc_DT_panel_adaptive(mesh.h, src, trg, atol, rtol, n_GL, max_depth, _d(out), C.byref(nl))
    return out, bool(hm), nl.value


def adaptive_panel_moments(mesh, src, pt, nt, atol, rtol, n_GL, max_depth):
    """``adaptive_panel_moments_inplace!`` (src/kernel/laplace3d_near_adaptive.jl:17-110)."""
    K = np.zeros(mesh.nq ** 2)
    hm = lib().orc_adaptive_panel_moments(mesh.h, src, _d(_cd(pt)), _d(_cd(nt)), atol, rtol, n_GL, max_depth, _d(K))
    return K, bool(hm)


def DT_corrections(mesh, ups, adp, adaptive_atol, adaptive_rtol=np.sqrt(np.finfo(float).eps), adaptive_n_GL=0,
                   adaptive_max_depth=20, nthreads=0):
    """``laplace3d_DT_corrections`` (src/kernel/laplace3d_near_upsampling.jl:127-276) as scipy CSC."""
    import scipy.sparse as sp
    s, keep = _nbr_handle(mesh, ups, adp)
    L = lib()
    h = L.orc_DT_corrections(mesh.h, C.cast(C.pointer(s), C.c_void_p), adaptive_atol, adaptive_rtol, adaptive_n_GL,
                             adaptive_max_depth, nthreads)
    nnz = int(L.orc_coo_nnz(h))
    r = np.zeros(nnz, dtype=np.int64)
    c = np.zeros(nnz, dtype=np.int64)
    v = np.zeros(nnz)
    L.orc_coo_copy(h, _l(r), _l(c), _d(v))
    hit = bool(L.orc_coo_hit_max(h))
    L.orc_coo_free(h)
    del keep
    M = sp.csc_matrix((v, (r, c)), shape=(mesh.n, mesh.n))
    M.sort_indices()
    M.hit_max = hit
    return M


def _csc_ptrs(Cm):
    if Cm is None:
        return None, None, None, ()
    colptr = np.ascontiguousarray(Cm.indptr, dtype=np.int64)
    rowidx = np.ascontiguousarray(Cm.indices, dtype=np.int64)
    vals = np.ascontiguousarray(Cm.data, dtype=np.float64)
    return colptr, rowidx, vals, (colptr, rowidx, vals)


def op_apply(mesh, x, Cm=None, nthreads=0):
    """Corrected operator action D^T x + C x + t .* x
    (src/kernel/laplace3d_near.jl:395-419 with the direct sum for the FMM)."""
    x = _cd(x)
    y = np.zeros(mesh.n)
    cp, ri, cv, keep = _csc_ptrs(Cm)
    lib().orc_op_apply(mesh.n, _d(mesh.pts), _d(mesh.nrm), _d(mesh.w), _d(mesh.diag()), _l(cp), _l(ri), _d(cv),
                       _d(x), _d(y), nthreads)
    return y


def gmres(mesh, b, Cm=None, atol=1e-6, rtol=1e-6, itmax=1000, nthreads=0, diag=None):
    """``solve_gmres`` (src/utils/linear_algebra.jl:3-5) on the corrected operator.
    Returns (x, iterations, residual estimate)."""
    b = _cd(b)
    x = np.zeros(mesh.n)
    res = C.c_double(0.0)
    cp, ri, cv, keep = _csc_ptrs(Cm)
    dg = _cd(mesh.diag() if diag is None else diag)
    it = lib().orc_gmres(mesh.n, _d(mesh.pts), _d(mesh.nrm), _d(mesh.w), _d(dg), _l(cp), _l(ri), _d(cv), _d(b),
                         _d(x), atol, rtol, itmax, nthreads, C.byref(res))
    return x, it, res.value
