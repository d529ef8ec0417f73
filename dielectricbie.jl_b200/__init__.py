"""B200-native drop-in for DielectricBIE.jl's layer-potential hot path.

Host-side mirror of the reference's Julia API (same names, argument meaning and
error behaviour) on top of the C ABI of ``libbie_b200.so``:

  geometry   single_dielectric_box3d, multi_dielectric_box3d, rect_panel3d_discretize,
             DielectricInterface, FlatPanel, PointSource, num_points, all_weights, eachpoint
  near field build_neighbor_list, laplace3d_DT_corrections
  operators  lhs_dielectric_box3d, lhs_dielectric_box3d_fmm3d(_corrected),
             batched_lhs_dielectric_box3d_fmm3d_corrected (GPU operators with mul!/@),
             rhs_dielectric_box3d, laplace3d_pottrg, dielectric_diagonal_scaling,
             laplace3d_pottrg_fmm3d_corrected_hcubature (near-accurate probe potentials)
  solvers    solve_gmres, solve_dielectric_box3d_block, gpu_solve, gpu_solve_sources

The mesher and the correction-block setup run on the host (as in the
reference); the direct sums, the correction apply and the Krylov iterations run
on the GPU. There is no CPU fallback: operator construction raises when no CUDA
device or no library is available.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _abi
from ._abi import BieError, NotConverged, check, dptr, i32ptr, iptr, lib

__all__ = [
    "PointSource", "FlatPanel", "DielectricInterface", "AdaptiveConfig", "gausslegendre", "best_grid_mn",
    "rect_panel3d_discretize", "single_dielectric_box3d", "multi_dielectric_box3d", "num_points", "all_weights",
    "eachpoint", "laplace3d_pot", "laplace3d_grad", "build_neighbor_list", "laplace3d_DT_corrections",
    "GPUDielectricOperator", "BatchedDielectricOperator", "lhs_dielectric_box3d", "lhs_dielectric_box3d_fmm3d",
    "lhs_dielectric_box3d_fmm3d_corrected", "batched_lhs_dielectric_box3d_fmm3d_corrected",
    "rhs_dielectric_box3d", "laplace3d_pottrg", "dielectric_diagonal_scaling", "solve_gmres",
    "solve_dielectric_box3d_block", "gpu_solve", "gpu_solve_sources", "polarization_energy", "BieError", "NotConverged",
    "laplace3d_pottrg_fmm3d_corrected_hcubature", "ProbePotentialOperator",
]

SQRT_EPS = math.sqrt(np.finfo(float).eps)


# ---------------------------------------------------------------------------
# Sources and panels (src/core/sources.jl:5-8, src/core/panels.jl:5-68)
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class PointSource:
    """``PointSource{T,3}(point, charge)`` (src/core/sources.jl:5-8)."""
    point: Tuple[float, float, float]
    charge: float


@dataclass
class FlatPanel:
    """``FlatPanel{T,3}`` (src/core/panels.jl:5-22): corners (a, b, c, d) anti-clockwise,
    tensor Gauss-Legendre nodes (b-a index outer, d-a index inner) and weights."""
    normal: Tuple[float, float, float]
    corners: np.ndarray  # (4, 3)
    is_edge: bool
    n_quad: int
    gl_xs: np.ndarray
    gl_ws: np.ndarray
    points: np.ndarray   # (n_quad^2, 3)
    weights: np.ndarray  # (n_quad^2,)
    bary_weights: np.ndarray = field(default=None)


@dataclass(frozen=True)
class AdaptiveConfig:
    """``AdaptiveConfig`` (src/kernel/laplace3d_near_adaptive.jl:3-12)."""
    atol: float
    rtol: float = SQRT_EPS
    n_GL: int = 0
    max_depth: int = 20


def gausslegendre(n: int):
    """Gauss-Legendre nodes (ascending) and weights, as FastGaussQuadrature.gausslegendre."""
    x = np.zeros(n)
    w = np.zeros(n)
    check(lib().bie_gausslegendre(int(n), dptr(x), dptr(w)))
    return x, w


def best_grid_mn(W: float, H: float, alpha: float):
    """``best_grid_mn`` (src/utils/best_grid.jl:120-126); ValueError like Julia's ArgumentError."""
    m, n = C.c_int(0), C.c_int(0)
    rc = lib().bie_best_grid(float(W), float(H), float(alpha), C.byref(m), C.byref(n))
    if rc != _abi.BIE_OK:
        raise ValueError(_abi.last_error())
    return m.value, n.value


def _bary_weights(x, w):
    n = len(x)
    lam = np.array([(1.0 if (n - 1 - i) % 2 == 0 else -1.0) * math.sqrt((1 - x[i] ** 2) * w[i] / 2) for i in range(n)])
    return lam / np.abs(lam).max()


def rect_panel3d_discretize(a, b, c, d, ns, ws, normal, is_edge: bool = False) -> FlatPanel:
    """``rect_panel3d_discretize`` (src/shape/box3d.jl:22-64)."""
    a, b, c, d = (np.asarray(v, dtype=np.float64) for v in (a, b, c, d))
    ns = np.asarray(ns, dtype=np.float64)
    ws = np.asarray(ws, dtype=np.float64)
    Lab, Lbc = np.linalg.norm(b - a), np.linalg.norm(c - b)
    if not (np.isclose(Lab, np.linalg.norm(d - c)) and np.isclose(Lbc, np.linalg.norm(a - d))):
        raise ValueError("Edges of the square are not equal")
    nrm = np.asarray(normal, dtype=np.float64)
    for e in (b - a, c - b, d - c, a - d):
        if abs(nrm @ e) >= 1e-10:
            raise ValueError("Normal is not perpendicular to the edges")
    cc = (((a + b) + c) + d) / 4
    q = len(ns)
    pts = np.array([(cc + (b - a) * (ns[i] / 2)) + (d - a) * (ns[j] / 2) for i in range(q) for j in range(q)])
    wts = np.array([ws[i] * ws[j] * Lab * Lbc / 4 for i in range(q) for j in range(q)])
    return FlatPanel(tuple(nrm), np.stack([a, b, c, d]), bool(is_edge), q, ns, ws, pts, wts, _bary_weights(ns, ws))


# ---------------------------------------------------------------------------
# DielectricInterface backed by a library mesh handle
# ---------------------------------------------------------------------------
class DielectricInterface:
    """``DielectricInterface`` (src/core/panels.jl:64-68): panels + per-panel eps_in/eps_out.

    Construct from FlatPanels, or through single_/multi_dielectric_box3d."""

    def __init__(self, panels: Optional[Sequence[FlatPanel]] = None, eps_in=None, eps_out=None, *, _handle=None):
        L = lib()
        if _handle is None:
            panels = list(panels)
            if not panels:
                raise ValueError("an interface needs at least one panel")
            nq = panels[0].n_quad
            if any(p.n_quad != nq for p in panels):
                raise NotImplementedError("panels with different n_quad are not supported")
            P = len(panels)
            corners = np.ascontiguousarray(np.stack([p.corners for p in panels]), dtype=np.float64)
            normals = np.ascontiguousarray([p.normal for p in panels], dtype=np.float64)
            ie = np.ascontiguousarray([int(p.is_edge) for p in panels], dtype=np.intc)
            ei = np.ascontiguousarray(np.broadcast_to(np.asarray(eps_in, dtype=np.float64), (P,)))
            eo = np.ascontiguousarray(np.broadcast_to(np.asarray(eps_out, dtype=np.float64), (P,)))
            h = C.c_void_p()
            check(L.bie_mesh_from_panels(P, nq, dptr(corners), dptr(normals), iptr(ie), dptr(ei), dptr(eo),
                                         C.byref(h)))
            _handle = h
        self._h = _handle
        n, P, nq = C.c_int64(0), C.c_int(0), C.c_int(0)
        check(L.bie_mesh_info(self._h, C.byref(n), C.byref(P), C.byref(nq)))
        self.n, self.npanels, self.n_quad = n.value, P.value, nq.value
        P, N = self.npanels, self.n
        self.corners = np.zeros((P, 4, 3))
        self.panel_normals = np.zeros((P, 3))
        self.is_edge = np.zeros(P, dtype=np.intc)
        self.eps_in = np.zeros(P)
        self.eps_out = np.zeros(P)
        self.points = np.zeros((N, 3))
        self.normals = np.zeros((N, 3))
        self.weights = np.zeros(N)
        self.diag = np.zeros(N)
        check(L.bie_mesh_copy(self._h, dptr(self.corners), dptr(self.panel_normals), iptr(self.is_edge),
                              dptr(self.eps_in), dptr(self.eps_out), dptr(self.points), dptr(self.normals),
                              dptr(self.weights), dptr(self.diag)))
        self._panels = None
        self._near: Dict[tuple, "_Near"] = {}
        self._geoms: Dict[tuple, "_Geom"] = {}

    def __del__(self):
        try:
            for g in self._geoms.values():
                g.close()
            lib().bie_mesh_destroy(self._h)
        except Exception:
            pass

    def __repr__(self):
        return f"DielectricInterface with {self.npanels} panels in Float64"

    @property
    def panels(self) -> List[FlatPanel]:
        if self._panels is None:
            x, w = gausslegendre(self.n_quad)
            lam = _bary_weights(x, w)
            q2 = self.n_quad ** 2
            self._panels = [
                FlatPanel(tuple(self.panel_normals[p]), self.corners[p], bool(self.is_edge[p]), self.n_quad, x, w,
                          self.points[p * q2:(p + 1) * q2], self.weights[p * q2:(p + 1) * q2], lam)
                for p in range(self.npanels)]
        return self._panels

    # cached near-field blocks and device geometries ----------------------------
    def near(self, max_order=8, up_tol=1e-9, correct_edges=True, adaptive: Optional[AdaptiveConfig] = None,
             nthreads=0, setup_device: Optional[int] = None) -> "_Near":
        """Near-field corrections (cached). setup_device: CUDA device for the adaptive blocks'
        moment sums (bitwise equal to the host's); None = device 0 when the library sees a
        CUDA device, else the host."""
        if setup_device is None:
            setup_device = 0 if _abi.device_count() > 0 else -1
        ad = adaptive or AdaptiveConfig(atol=up_tol)
        key = (int(max_order), float(up_tol), bool(correct_edges), ad, int(nthreads))
        if key not in self._near:
            self._near[key] = _Near(self, max_order, up_tol, correct_edges, ad, nthreads, setup_device)
        return self._near[key]

    def geom(self, near: Optional["_Near"], device: int = 0) -> "_Geom":
        key = (id(near) if near is not None else None, device)
        if key not in self._geoms:
            if near is not None and near.released:
                raise RuntimeError("the near-field blocks' host values were released (keep_host_blocks=False); "
                                   "a geometry on another device needs them: build that operator first")
            self._geoms[key] = _Geom(self, near, device)
        return self._geoms[key]


def num_points(itf: DielectricInterface) -> int:
    """``num_points`` (src/core/panels.jl:117)."""
    return itf.n


def all_weights(itf: DielectricInterface) -> np.ndarray:
    """``all_weights`` (src/core/panels.jl:118)."""
    return itf.weights.copy()


def eachpoint(itf: DielectricInterface):
    """Interface iteration order (src/core/panels.jl:87-115): (global_idx, panel_idx, point, normal, weight)."""
    q2 = itf.n_quad ** 2
    for i in range(itf.n):
        yield i, i // q2, itf.points[i], itf.normals[i], itf.weights[i]


def single_dielectric_box3d(Lx, Ly, Lz, n_quad, l_ec, eps_in, eps_out, T=float, *, alpha=math.sqrt(2.0)):
    """``single_dielectric_box3d`` (src/shape/box3d_single.jl:49-70)."""
    h = C.c_void_p()
    check(lib().bie_mesh_single_box(float(Lx), float(Ly), float(Lz), int(n_quad), float(l_ec), float(eps_in),
                                    float(eps_out), float(alpha), C.byref(h)))
    return DielectricInterface(_handle=h)


def multi_dielectric_box3d(n_quad, l_ec, boxes, epses, eps_out=1.0, *, alpha=math.sqrt(2.0)):
    """``multi_dielectric_box3d`` (src/shape/box3d_multi.jl:358-386). boxes: sequence of
    dicts/tuples (center, Lx, Ly, Lz)."""
    cs, ds = [], []
    for b in boxes:
        if isinstance(b, dict):
            cs.append(b["center"]); ds.append((b["Lx"], b["Ly"], b["Lz"]))
        else:
            cs.append(b[0]); ds.append(tuple(b[1:4]))
    if len(cs) != len(epses):
        raise ValueError("Number of boxes must match number of permittivities")
    c = np.ascontiguousarray(cs, dtype=np.float64)
    d = np.ascontiguousarray(ds, dtype=np.float64)
    e = np.ascontiguousarray(epses, dtype=np.float64)
    h = C.c_void_p()
    check(lib().bie_mesh_multi_box(int(n_quad), float(l_ec), len(e), dptr(c), dptr(d), dptr(e), float(eps_out),
                                   float(alpha), C.byref(h)))
    return DielectricInterface(_handle=h)


def laplace3d_pot(src, trg) -> float:
    """``laplace3d_pot`` (src/kernel/laplace3d.jl:1-7), host scalar."""
    r = np.linalg.norm(np.asarray(src, float) - np.asarray(trg, float))
    return (1.0 / r) / (4 * math.pi)


def laplace3d_grad(src, trg, n) -> float:
    """``laplace3d_grad`` (src/kernel/laplace3d.jl:9-15), host scalar."""
    src, trg, n = (np.asarray(v, float) for v in (src, trg, n))
    d = trg - src
    ir = 1.0 / math.sqrt(float(d @ d))
    return float(n @ (ir ** 3 * d)) / (4 * math.pi)


# ---------------------------------------------------------------------------
# Near field (src/kernel/laplace3d_near.jl:240-392, laplace3d_near_upsampling.jl:127-276)
# ---------------------------------------------------------------------------
class _Near:
    def __init__(self, itf, max_order, up_tol, correct_edges, ad: AdaptiveConfig, nthreads, setup_device=-1):
        o = _abi.NearOpts()
        lib().bie_near_opts_default(C.byref(o))
        o.max_order, o.up_tol, o.correct_edges = int(max_order), float(up_tol), int(bool(correct_edges))
        o.adaptive_atol, o.adaptive_rtol = float(ad.atol), float(ad.rtol)
        o.adaptive_n_GL, o.adaptive_max_depth, o.nthreads = int(ad.n_GL), int(ad.max_depth), int(nthreads)
        o.device = int(setup_device)
        h = C.c_void_p()
        check(lib().bie_near_build(itf._h, C.byref(o), C.byref(h)))
        self._h = h
        nbl, nb, nu, na, hm = C.c_int64(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib().bie_near_info(h, C.byref(nbl), C.byref(nb), C.byref(nu), C.byref(na), C.byref(hm)))
        self.nblocks, self.nb, self.hit_max_depth = nbl.value, nb.value, bool(hm.value)
        self.rowptr = np.zeros(itf.npanels + 1, dtype=np.int32)
        self.col = np.zeros(self.nblocks, dtype=np.int32)
        self._val = None  # the block values stay in the library's copy until asked for
        check(lib().bie_near_copy(h, i32ptr(self.rowptr), i32ptr(self.col), None, None, None, None, None, None))
        self._npairs = (nu.value, na.value)
        self._ad = ad
        self._pairs = None  # the pair lists, copied out of the library on first use
        self.n = itf.n
        self.values_geom = None  # set once the host values are released: the geometry holding them

    def _pair_lists(self):
        if self._pairs is None:
            nu, na = self._npairs
            ui, uj, up = (np.zeros(nu, dtype=np.int32) for _ in range(3))
            ai, aj = (np.zeros(na, dtype=np.int32) for _ in range(2))
            check(lib().bie_near_copy(self._h, None, None, None, i32ptr(ui), i32ptr(uj), i32ptr(up), i32ptr(ai),
                                      i32ptr(aj)))
            self._pairs = ({(int(i), int(j)): int(p) for i, j, p in zip(ui, uj, up)},
                           {(int(i), int(j)): self._ad for i, j in zip(ai, aj)})
        return self._pairs

    @property
    def upsample(self) -> dict:
        """(source panel, target panel) -> upsampling order, 0-based."""
        return self._pair_lists()[0]

    @property
    def adaptive(self) -> dict:
        """(source panel, target panel) -> AdaptiveConfig of the touching pairs, 0-based."""
        return self._pair_lists()[1]

    @property
    def released(self) -> bool:
        return self.values_geom is not None

    def release_host_values(self, geom: "_Geom"):
        """Frees the library's host copy of the block values (``bie_near_release_values``);
        ``geom``, a device geometry built from these blocks, holds them from then on and
        ``val`` reads them back from it."""
        if self.released:
            return
        check(lib().bie_near_release_values(self._h))
        self.values_geom = geom

    @property
    def val(self) -> np.ndarray:
        """Correction block values (nblocks x nb x nb, each block column-major), copied out
        of the library on first use (out of the device geometry once the host copy was
        released); a geometry that is only solved on the device never holds a second host
        copy of its blocks."""
        if self._val is None:
            v = np.zeros(self.nblocks * self.nb * self.nb)
            if self.released:
                check(lib().bie_geom_near_values(self.values_geom._h, dptr(v), v.size))
            else:
                check(lib().bie_near_copy(self._h, None, None, dptr(v), None, None, None, None, None))
            self._val = v
        return self._val

    def __del__(self):
        try:
            lib().bie_near_destroy(self._h)
        except Exception:
            pass

    def to_scipy(self):
        """The correction matrix C (N x N) as scipy.sparse.bsr (host copy, for inspection/tests)."""
        import scipy.sparse as sp
        nb = self.nb
        blocks = self.val.reshape(self.nblocks, nb, nb).transpose(0, 2, 1)  # stored column-major
        return sp.bsr_matrix((blocks, self.col, self.rowptr), shape=(self.n, self.n))


def build_neighbor_list(interface: DielectricInterface, max_order: int, atol: float, *, correct_edges: bool = False,
                        adaptive_cfg: Optional[AdaptiveConfig] = None):
    """``build_neighbor_list`` (src/kernel/laplace3d_near.jl:240-392). Returns (upsample, adaptive)
    dicts keyed by 0-based (source panel, target panel)."""
    nr = interface.near(max_order, atol, correct_edges, adaptive_cfg)
    return nr.upsample, nr.adaptive


def laplace3d_DT_corrections(interface: DielectricInterface, *, max_order=8, up_tol=1e-9, correct_edges=True,
                             adaptive_cfg: Optional[AdaptiveConfig] = None):
    """``laplace3d_DT_corrections`` (src/kernel/laplace3d_near_upsampling.jl:272-276) as a sparse matrix."""
    return interface.near(max_order, up_tol, correct_edges, adaptive_cfg).to_scipy()


# ---------------------------------------------------------------------------
# GPU geometry and operators
# ---------------------------------------------------------------------------
class _Geom:
    def __init__(self, itf: DielectricInterface, near: Optional[_Near], device: int):
        h = C.c_void_p()
        check(lib().bie_geom_create_from_mesh(itf._h, near._h if near is not None else None, int(device),
                                              C.byref(h)))
        self._h = h
        self.n = itf.n

    def close(self):
        if self._h:
            lib().bie_geom_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(lib().bie_geom_stream(self._h) or 0)


def _as_cols(X, n):
    X = np.asarray(X, dtype=np.float64)
    vec = X.ndim == 1
    Xf = np.asfortranarray(X.reshape(n, -1) if vec else X)
    if Xf.shape[0] != n:
        raise ValueError(f"dimension mismatch: expected {n} rows, got {Xf.shape[0]}")
    return Xf, vec


class GPUDielectricOperator:
    """The dielectric BIE operator A = D^T + C + diag(t_P) on the GPU.

    Drop-in for the LinearMaps/BatchedDielectricOperator the reference's solvers
    accept (size, eltype, mul!; src/solver/multi_rhs.jl:46-141), with the FMM
    replaced by the exact direct sum. ``precision`` selects the arithmetic of the
    direct sum: "fp64" (plain), "fp32" (FP64 tile partials) or "bf16x3"
    (tensor-core RHS contraction; FP32 CUDA-core sum for k = 1, 2, 4). Corrections and diagonal stay FP64."""

    def __init__(self, interface: DielectricInterface, *, precision: str = "fp64", corrections: bool = True,
                 up_tol: float = 1e-9, max_order: int = 8, correct_edges: bool = True,
                 adaptive_cfg: Optional[AdaptiveConfig] = None, device: int = 0, keep_host_blocks: bool = True,
                 nthreads: int = 0):
        if precision not in _abi.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_abi.PRECISIONS)}")
        self.interface = interface
        self.precision = precision
        self.near = interface.near(max_order, up_tol, correct_edges, adaptive_cfg, nthreads) if corrections else None
        self.geom = interface.geom(self.near, device)
        if self.near is not None and not keep_host_blocks:
            # the blocks live on the device only (a server's many resident geometries)
            self.near.release_host_values(self.geom)
        self.n = interface.n
        self.shape = (self.n, self.n)
        self.dtype = np.float64

    def __repr__(self):
        c = "corrected" if self.near is not None else "uncorrected"
        return f"GPUDielectricOperator({self.n}x{self.n}, {self.precision}, {c})"

    def size(self, d=None):
        return self.shape if d is None else self.shape[d - 1]

    def eltype(self):
        return np.float64

    def mul(self, X, *, precision: Optional[str] = None, flags: int = 0):
        """``mul!(Y, op, X)``: X is (N,) or (N, k) column-major like Julia."""
        Xf, vec = _as_cols(X, self.n)
        k = Xf.shape[1]
        Y = np.zeros((self.n, k), order="F")
        p = _abi.PRECISIONS[precision or self.precision]
        check(lib().bie_matvec(self.geom._h, dptr(Xf), dptr(Y), k, p, flags))
        return Y[:, 0] if vec else Y

    def __matmul__(self, X):
        return self.mul(X)

    __mul__ = __matmul__

    def matvec_device(self, dX_ptr: int, dY_ptr: int, k: int, stream: int = 0, precision: Optional[str] = None,
                      flags: int = 0):
        """Device-pointer matvec (node-major N x k) ordered on ``stream``."""
        p = _abi.PRECISIONS[precision or self.precision]
        check(lib().bie_matvec_device(self.geom._h, C.c_void_p(dX_ptr), C.c_void_p(dY_ptr), k, p, flags,
                                      C.c_void_p(stream)))


BatchedDielectricOperator = GPUDielectricOperator


def lhs_dielectric_box3d(interface: DielectricInterface, *, device: int = 0):
    """``lhs_dielectric_box3d`` (src/solver/dielectric_box3d.jl:1-17): D^T (j != i) + diag(t_P),
    no near-field correction, as a GPU operator (FP64)."""
    return GPUDielectricOperator(interface, corrections=False, device=device)


def lhs_dielectric_box3d_fmm3d(interface: DielectricInterface, tol: float = 1e-6, *, device: int = 0):
    """``lhs_dielectric_box3d_fmm3d`` (src/solver/dielectric_box3d.jl:20-44); the FMM is replaced by the
    exact direct sum, so ``tol`` has no effect."""
    return GPUDielectricOperator(interface, corrections=False, device=device)


def lhs_dielectric_box3d_fmm3d_corrected(interface: DielectricInterface, fmm_tol: float, up_tol: float,
                                         max_order: int, *, correct_edges: bool = True,
                                         adaptive_atol: Optional[float] = None, adaptive_rtol: float = SQRT_EPS,
                                         adaptive_n_GL: int = 0, adaptive_max_depth: int = 20,
                                         precision: str = "fp64", device: int = 0, keep_host_blocks: bool = True,
                                         nthreads: int = 0):
    """``lhs_dielectric_box3d_fmm3d_corrected`` (src/solver/dielectric_box3d.jl:48-92).
    keep_host_blocks=False frees the host copy of the correction blocks once they are on the
    device (they are read back from there on request); nthreads bounds the host threads of
    the near-field set-up (0 = all)."""
    ad = AdaptiveConfig(up_tol if adaptive_atol is None else adaptive_atol, adaptive_rtol, adaptive_n_GL,
                        adaptive_max_depth)
    return GPUDielectricOperator(interface, precision=precision, corrections=True, up_tol=up_tol,
                                 max_order=max_order, correct_edges=correct_edges, adaptive_cfg=ad, device=device,
                                 keep_host_blocks=keep_host_blocks, nthreads=nthreads)


def batched_lhs_dielectric_box3d_fmm3d_corrected(interface, fmm_tol, up_tol, max_order, **kw):
    """``batched_lhs_dielectric_box3d_fmm3d_corrected`` (src/solver/multi_rhs.jl:60-100)."""
    return lhs_dielectric_box3d_fmm3d_corrected(interface, fmm_tol, up_tol, max_order, **kw)


def _point_sources(sources, eps_src):
    if isinstance(sources, PointSource):
        sources = [sources]
    sources = list(sources)
    k = len(sources)
    src = np.ascontiguousarray([s.point for s in sources], dtype=np.float64).reshape(k, 3)
    q = np.ascontiguousarray([s.charge for s in sources], dtype=np.float64)
    eps = np.ascontiguousarray(np.broadcast_to(np.asarray(eps_src, dtype=np.float64), (k,)))
    return src, q, eps


def rhs_dielectric_box3d(interface: DielectricInterface, ps, eps_src, *, device: int = 0):
    """``rhs_dielectric_box3d(itf, ::PointSource, eps_src)`` (src/solver/dielectric_box3d.jl:95-104),
    computed on the GPU. A list of sources gives the N x k block right-hand side."""
    single = isinstance(ps, PointSource)
    src, q, eps = _point_sources(ps, eps_src)
    k = len(q)
    g = interface.geom(None, device)
    F = np.zeros((interface.n, k), order="F")
    check(lib().bie_rhs_point(g._h, dptr(src), dptr(q), dptr(eps), k, dptr(F)))
    return F[:, 0] if single else F


class _PotentialOperator:
    def __init__(self, interface, targets, device):
        T = np.asarray(targets, dtype=np.float64)
        if T.ndim == 2 and T.shape[0] == 3 and T.shape[1] != 3:
            T = T.T
        self.T = np.ascontiguousarray(T.reshape(-1, 3))
        self.geom = interface.geom(None, device)
        self.n = interface.n
        self.shape = (self.T.shape[0], self.n)

    def __matmul__(self, S):
        Sf, vec = _as_cols(S, self.n)
        k = Sf.shape[1]
        M = self.T.shape[0]
        phi = np.zeros((M, k), order="F")
        check(lib().bie_potential(self.geom._h, dptr(Sf), k, dptr(self.T), M, dptr(phi)))
        return phi[:, 0] if vec else phi

    __mul__ = __matmul__


def laplace3d_pottrg(interface: DielectricInterface, targets, *, device: int = 0):
    """``laplace3d_pottrg`` (src/kernel/laplace3d.jl:69-82): the M x N single-layer map at targets,
    applied on the GPU (``op @ sigma``). targets: (M, 3) or 3 x M."""
    return _PotentialOperator(interface, targets, device)


def _targets_3xM(targets) -> np.ndarray:
    T = np.asarray(targets, dtype=np.float64)
    if T.ndim == 2 and T.shape[0] == 3 and T.shape[1] != 3:
        T = T.T
    return np.ascontiguousarray(T.reshape(-1, 3))


class ProbePotentialOperator:
    """Near-accurate potentials at probe points, the M x N operator of
    ``laplace3d_pottrg_fmm3d_corrected_hcubature`` (src/kernel/laplace3d_near_hcubature.jl:278-316):
    phi = (S_refined + C) P sigma, with the panels near the probes refined, P the
    prolongation onto the refined nodes, S_refined their smooth-quadrature potential (GPU
    direct sum) and C the adaptive-quadrature corrections of probes near refined non-edge
    panels. ``op @ Sigma`` applies it on the GPU; device < 0 keeps only the host set-up."""

    def __init__(self, interface: DielectricInterface, targets, hcubature_atol: float, range_factor: float,
                 device: int = 0):
        self.T = _targets_3xM(targets)
        self.n = interface.n
        self.shape = (self.T.shape[0], self.n)
        h = C.c_void_p()
        check(lib().bie_probe_create(interface._h, dptr(self.T), self.T.shape[0], float(hcubature_atol),
                                     float(range_factor), int(device), C.byref(h)))
        self._h = h

    def info(self) -> dict:
        v = [C.c_int64(), C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()]
        check(lib().bie_probe_info(self._h, *[C.byref(x) for x in v]))
        keys = ["n_refined", "npanels_refined", "nnz_prolongation", "nnz_corrections", "ncubatures", "capped"]
        return {k: x.value for k, x in zip(keys, v)}

    def refinement(self) -> dict:
        """The host operator: parent coarse panel and split flag per refined panel, refined
        corners (R, 4, 3), nodes (n_ref, 3) and weights, and P (n_ref x N) and C (M x n_ref)
        as CSR triples (rowptr, col, val)."""
        inf = self.info()
        R, nr, nnp, nnc = inf["npanels_refined"], inf["n_refined"], inf["nnz_prolongation"], inf["nnz_corrections"]
        M = self.T.shape[0]
        out = {"parent": np.zeros(R, dtype=np.int32), "from_split": np.zeros(R, dtype=np.int32),
               "corners": np.zeros((max(R, 1), 4, 3)), "points": np.zeros((max(nr, 1), 3)),
               "weights": np.zeros(max(nr, 1)), "prow": np.zeros(nr + 1, dtype=np.int64),
               "pcol": np.zeros(max(nnp, 1), dtype=np.int32), "pval": np.zeros(max(nnp, 1)),
               "crow": np.zeros(M + 1, dtype=np.int64), "ccol": np.zeros(max(nnc, 1), dtype=np.int32),
               "cval": np.zeros(max(nnc, 1))}
        i64 = C.POINTER(C.c_int64)
        check(lib().bie_probe_copy(self._h, i32ptr(out["parent"]), i32ptr(out["from_split"]), dptr(out["corners"]),
                                   dptr(out["points"]), dptr(out["weights"]), out["prow"].ctypes.data_as(i64),
                                   i32ptr(out["pcol"]), dptr(out["pval"]), out["crow"].ctypes.data_as(i64),
                                   i32ptr(out["ccol"]), dptr(out["cval"])))
        out["from_split"] = out["from_split"].astype(bool)
        out["corners"], out["points"], out["weights"] = out["corners"][:R], out["points"][:nr], out["weights"][:nr]
        out["pcol"], out["pval"], out["ccol"], out["cval"] = (out["pcol"][:nnp], out["pval"][:nnp],
                                                              out["ccol"][:nnc], out["cval"][:nnc])
        return out

    def __matmul__(self, S):
        Sf, vec = _as_cols(S, self.n)
        k = Sf.shape[1]
        M = self.T.shape[0]
        phi = np.zeros((M, k), order="F")
        check(lib().bie_probe_apply(self._h, dptr(Sf), k, dptr(phi)))
        return phi[:, 0] if vec else phi

    __mul__ = __matmul__

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().bie_probe_destroy(h)
            except Exception:
                pass
            self._h = None


def laplace3d_pottrg_fmm3d_corrected_hcubature(interface: DielectricInterface, targets, fmm_tol: float,
                                               hcubature_atol: float, range_factor: float = 5.0, *,
                                               device: int = 0) -> ProbePotentialOperator:
    """``laplace3d_pottrg_fmm3d_corrected_hcubature(interface, targets, fmm_tol, hcubature_atol,
    range_factor)`` (src/kernel/laplace3d_near_hcubature.jl:278-316). The far part is the exact
    direct sum, so fmm_tol (the FMM's tolerance in the reference) has nothing to set."""
    del fmm_tol
    return ProbePotentialOperator(interface, targets, hcubature_atol, range_factor, device)


def polarization_energy(interface: DielectricInterface, Sigma, sources, *, device: int = 0):
    """W_c = 1/2 q_c S[Sigma[:, c]](x_c) for point sources (a quantity the reference
    does not define; evaluated with the same single-layer sum)."""
    src, q, _ = _point_sources(sources, 1.0)
    Sf, _ = _as_cols(Sigma, interface.n)
    k = Sf.shape[1]
    W = np.zeros(k)
    check(lib().bie_energy(interface.geom(None, device)._h, dptr(Sf), k, dptr(src), dptr(q), dptr(W)))
    return W


def dielectric_diagonal_scaling(interface: DielectricInterface) -> np.ndarray:
    """``dielectric_diagonal_scaling`` (src/solver/multi_rhs.jl:234-247): 1 / t_P per node."""
    return 1.0 / interface.diag


@dataclass
class SolveStats:
    iterations: int
    outer: int
    fp64_matvecs: int
    lowp_matvecs: int
    solved: bool
    max_rel_resid: float
    seconds: float
    col_iterations: np.ndarray
    col_resid: np.ndarray


def _solve_opts(op, rtol, atol, itmax, restart, precision, inner_rtol, max_outer, precondition, check_every,
                block=False):
    o = _abi.SolveOpts()
    lib().bie_solve_opts_default(C.byref(o))
    o.atol, o.rtol, o.itmax, o.restart = float(atol), float(rtol), int(itmax), int(restart)
    o.precision = _abi.PRECISIONS[precision or op.precision]
    o.inner_rtol, o.max_outer, o.precondition, o.check_every = float(inner_rtol), int(max_outer), int(precondition), int(check_every)
    o.block = int(bool(block))
    if op.near is None:
        o.flags = 0
    return o


def gpu_solve(op: GPUDielectricOperator, F, *, rtol: float = 1e-10, atol: float = 0.0, itmax: int = 500,
              restart: int = 200, precision: Optional[str] = None, inner_rtol: float = 1e-6, max_outer: int = 8,
              precondition: bool = False, check_every: int = 1, raise_on_noconv: bool = False, block: bool = False):
    """Solve A Sigma = F on the device. Returns (Sigma, SolveStats). block=True runs block GMRES
    (one Krylov space shared by the columns, as Krylov.block_gmres) for 2 to 64 columns; wider
    blocks run one Arnoldi process per column, which is faster with this library's kernels."""
    Ff, vec = _as_cols(F, op.n)
    k = Ff.shape[1]
    o = _solve_opts(op, rtol, atol, itmax, restart, precision, inner_rtol, max_outer, precondition, check_every,
                    block)
    S, stats = _run_solve(op, k, raise_on_noconv,
                          lambda S, st: lib().bie_solve(op.geom._h, dptr(Ff), dptr(S), k, C.byref(o), C.byref(st)))
    return (S[:, 0] if vec else S), stats


def _run_solve(op, k, raise_on_noconv, call):
    ci = np.zeros(k, dtype=np.intc)
    cr = np.zeros(k)
    st = _abi.Stats()
    st.col_iterations = ci.ctypes.data_as(C.POINTER(C.c_int))
    st.col_resid = cr.ctypes.data_as(C.POINTER(C.c_double))
    S = np.zeros((op.n, k), order="F")
    rc = call(S, st)
    if rc not in (_abi.BIE_OK, _abi.BIE_ENOCONV) or (rc == _abi.BIE_ENOCONV and raise_on_noconv):
        check(rc)
    stats = SolveStats(st.iterations, st.outer, st.fp64_matvecs, st.lowp_matvecs, bool(st.converged),
                       st.max_rel_resid, st.seconds, ci.copy(), cr.copy())
    return S, stats


def gpu_solve_sources(op: GPUDielectricOperator, sources, eps_src, *, rtol: float = 1e-10, atol: float = 0.0,
                      itmax: int = 500, restart: int = 200, precision: Optional[str] = None, inner_rtol: float = 1e-6,
                      max_outer: int = 8, precondition: bool = False, check_every: int = 1,
                      raise_on_noconv: bool = False, block: bool = False):
    """rhs_dielectric_box3d for point sources and the block solve in one call (C-ABI
    ``bie_solve_point``): the right-hand sides are built on the device, so only the sources
    go to the GPU and only Sigma comes back. Returns (Sigma N x k, SolveStats)."""
    src, q, eps = _point_sources(sources, eps_src)
    k = len(q)
    o = _solve_opts(op, rtol, atol, itmax, restart, precision, inner_rtol, max_outer, precondition, check_every,
                    block)
    return _run_solve(op, k, raise_on_noconv,
                      lambda S, st: lib().bie_solve_point(op.geom._h, dptr(src), dptr(q), dptr(eps), k, dptr(S),
                                                          C.byref(o), C.byref(st)))


def tuned_launch(op: "GPUDielectricOperator", family: str, k: int, pieces: int = 2):
    """The autotuned launch configuration the library chose for an operator's direct sum:
    family "tensor_core" (columns = min(k, 128)) or "fp64" (columns = min(k, 64)). Every width
    that runs the same kernel instance (a multiple of 16 for "tensor_core"; 8, 16, 32 or 64
    for "fp64") shares one entry. Returns dict(nsplit, ctas_per_sm, ms) or None when nothing
    was tuned yet."""
    fam, cols, pc = (0, min(k, 128), pieces) if family == "tensor_core" else (1, min(k, 64), 0)
    ns, ct, ms = C.c_int32(0), C.c_int32(0), C.c_double(0.0)
    rc = lib().bie_tuning_read(op.geom._h, fam, cols, pc, C.byref(ns), C.byref(ct), C.byref(ms))
    if rc != _abi.BIE_OK:
        return None
    return {"nsplit": ns.value, "ctas_per_sm": ct.value, "ms": ms.value}


class SolveServer:
    """Request server with continuous batching (C-ABI ``bie_server_*``).

    ``submit(op, F, ...)`` queues a block solve of F (N x k) on the operator's
    device-resident geometry and returns a ticket; ``result(ticket)`` waits for it and
    returns (Sigma, SolveStats, latency_ms). Up to ``max_slots`` block solves run at
    once, each on its geometry's stream; queued requests for the same geometry and
    options are merged into one block solve of at most ``max_batch_rhs`` columns;
    admission also respects an HBM budget (``hbm_fraction`` of the free memory).
    Point-source batches of up to ``max_group`` different geometries (split-BF16 precision)
    run together as one group solve, their direct sums in one launch per iteration.
    An operator handed to a server must not be used directly until its requests
    have been collected."""

    def __init__(self, *, max_slots: int = 4, max_batch_rhs: int = 128, hbm_fraction: float = 0.8, device: int = 0,
                 max_group: int = 8):
        o = _abi.ServerOpts()
        lib().bie_server_opts_default(C.byref(o))
        o.max_slots, o.max_batch_rhs, o.hbm_fraction, o.device = int(max_slots), int(max_batch_rhs), \
            float(hbm_fraction), int(device)
        o.max_group = int(max_group)
        h = C.c_void_p()
        check(lib().bie_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self._shapes = {}

    def submit(self, op: GPUDielectricOperator, F, *, rtol: float = 1e-10, atol: float = 0.0, itmax: int = 500,
               restart: int = 200, precision: Optional[str] = None, inner_rtol: float = 1e-6, max_outer: int = 8,
               precondition: bool = False, check_every: int = 1, block: bool = False) -> int:
        Ff, vec = _as_cols(F, op.n)
        k = Ff.shape[1]
        o = _solve_opts(op, rtol, atol, itmax, restart, precision, inner_rtol, max_outer, precondition, check_every,
                    block)
        t = C.c_uint64(0)
        check(lib().bie_server_submit(self._h, op.geom._h, dptr(Ff), k, C.byref(o), C.byref(t)))
        self._shapes[t.value] = (op.n, k, vec)
        return t.value

    def submit_sources(self, op: GPUDielectricOperator, sources, eps_src, *, rtol: float = 1e-10, atol: float = 0.0,
                       itmax: int = 500, restart: int = 200, precision: Optional[str] = None,
                       inner_rtol: float = 1e-6, max_outer: int = 8, precondition: bool = False,
                       check_every: int = 1, block: bool = False) -> int:
        """Queues the block solve of point-source right-hand sides (C-ABI
        ``bie_server_submit_point``): only the sources are held until the batch runs, which
        builds the right-hand sides on the device. The result is N x k as for submit()."""
        src, q, eps = _point_sources(sources, eps_src)
        k = len(q)
        o = _solve_opts(op, rtol, atol, itmax, restart, precision, inner_rtol, max_outer, precondition, check_every,
                    block)
        t = C.c_uint64(0)
        check(lib().bie_server_submit_point(self._h, op.geom._h, dptr(src), dptr(q), dptr(eps), k, C.byref(o),
                                            C.byref(t)))
        self._shapes[t.value] = (op.n, k, False)
        return t.value

    def result(self, ticket: int, timeout_ms: int = -1, *, sigma: bool = True):
        """(Sigma, SolveStats, latency_ms) once the request finished, else None after timeout_ms.
        sigma=False leaves Sigma out (None): the server drops it, nothing N x k is copied."""
        n, k, vec = self._shapes[ticket]
        S = np.zeros((n, k), order="F") if sigma else None
        ci = np.zeros(k, dtype=np.intc)
        cr = np.zeros(k)
        st = _abi.Stats()
        st.col_iterations = ci.ctypes.data_as(C.POINTER(C.c_int))
        st.col_resid = cr.ctypes.data_as(C.POINTER(C.c_double))
        lat = C.c_double(0.0)
        done = C.c_int(0)
        rc = lib().bie_server_poll(self._h, ticket, int(timeout_ms), dptr(S) if S is not None else None,
                                   C.byref(st), C.byref(lat), C.byref(done))
        if rc not in (_abi.BIE_OK, _abi.BIE_ENOCONV):
            del self._shapes[ticket]
            check(rc)
        if not done.value:
            return None
        del self._shapes[ticket]
        stats = SolveStats(st.iterations, st.outer, st.fp64_matvecs, st.lowp_matvecs, rc == _abi.BIE_OK,
                           st.max_rel_resid, st.seconds, ci, cr)
        if S is None:
            return None, stats, lat.value
        return (S[:, 0] if vec else S), stats, lat.value

    def counters(self) -> dict:
        c = _abi.ServerCounters()
        check(lib().bie_server_counters_read(self._h, C.byref(c)))
        return {f: getattr(c, f) for f, _ in c._fields_}

    def close(self):
        if self._h:
            lib().bie_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_gmres(A: GPUDielectricOperator, b, atol: float = 1e-6, rtol: float = 1e-6, itmax: int = 1000):
    """``solve_gmres`` (src/utils/linear_algebra.jl:3-5): GMRES from x0 = 0 with stopping rule
    ||r|| <= atol + rtol ||b||, run on the device. Like the reference, returns x even when
    itmax is reached."""
    if not isinstance(A, GPUDielectricOperator):
        raise TypeError("solve_gmres expects a GPUDielectricOperator")
    x, _ = gpu_solve(A, b, rtol=rtol, atol=atol, itmax=itmax, restart=min(itmax, 400))
    return x


def solve_dielectric_box3d_block(interface: DielectricInterface, sources, eps_src=None, *, fmm_tol: float = 1e-9,
                                 up_tol: float = 1e-9, max_order: int = 8, rtol: float = 1e-10, atol: float = 0.0,
                                 itmax: int = 500, precondition: bool = True, correct_edges: bool = True,
                                 precision: str = "fp64", device: int = 0, block: bool = True, **kw):
    """``solve_dielectric_box3d_block`` (src/solver/multi_rhs.jl:270-286) for PointSource right-hand
    sides (the reference takes VolumeSources; the operator is the same). eps_src defaults to each
    panel's eps_in of the first panel (source inside a single box). block=True (the default) solves
    up to 64 columns in one block Krylov space, as the reference's Krylov.block_gmres (wider blocks
    run one Arnoldi process per column, faster here); block=False runs one Arnoldi process per
    column. Returns (Sigma, stats)."""
    op = batched_lhs_dielectric_box3d_fmm3d_corrected(interface, fmm_tol, up_tol, max_order,
                                                      correct_edges=correct_edges, precision=precision,
                                                      device=device)
    if eps_src is None:
        eps_src = float(interface.eps_in[0])
    return gpu_solve_sources(op, list(sources), eps_src, rtol=rtol, atol=atol, itmax=itmax,
                             precondition=precondition, block=block, **kw)
