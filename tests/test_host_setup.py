"""Host side of libbie_b200 on CPU: the C ABI loads and exports what the header
declares, and the library's mesher and near-field builder (the set-up the
device operator is built from) agree with the oracle.

Mesh: bit-exact (same arithmetic order). Neighbour lists: identical pairs and
upsampling orders. Correction blocks: equal to the FP64 rounding level (the two
codes share the algorithm, not the summation order of every moment).
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bie_b200.h")

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bie_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_are_exported(bie):
    from dielectricbie_jl_b200 import _abi
    declared = header_functions()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], check=True, capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT (bie_[a-z0-9_]+)$", out, flags=re.M))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    # the ctypes binding declares a signature for every one of them
    assert sorted(_abi.EXPORTS) == declared
    L = _abi.lib()
    for f in declared:
        assert getattr(L, f) is not None


def test_library_loads_without_gpu(bie):
    from dielectricbie_jl_b200 import _abi
    assert _abi.version()
    assert _abi.device_count() >= 0


@pytest.mark.parametrize("cfg", [CFG1, (1.5, 1.0, 0.8, 6, 0.08, 4.0, 1.0), (1.0, 2.0, 3.0, 2, 10.0, 2.0, 1.0)])
def test_mesh_single_box_bit_exact(bie, orc, cfg):
    itf = bie.single_dielectric_box3d(*cfg)
    m = orc.Mesh.single_box(*cfg)
    assert itf.n == m.n and itf.npanels == m.npanels
    assert np.array_equal(itf.points, m.pts)
    assert np.array_equal(itf.normals, m.nrm)
    assert np.array_equal(itf.weights, m.w)
    assert np.array_equal(itf.corners, m.corners)
    assert np.array_equal(itf.is_edge, m.is_edge)
    assert np.array_equal(itf.diag, m.diag())


def test_mesh_multi_box_bit_exact(bie, orc):
    centers = [(0.0, 0.0, 0.0), (0.7, 0.0, 0.0), (0.0, 0.7, 0.0), (0.35, 0.35, 0.7)]
    dims = [(0.5, 0.5, 0.5)] * 4
    eps = [4.0, 2.0, 4.0, 8.0]
    itf = bie.multi_dielectric_box3d(4, 0.1, [{"center": c, "Lx": d[0], "Ly": d[1], "Lz": d[2]}
                                               for c, d in zip(centers, dims)], eps, 1.0)
    m = orc.Mesh.multi_box(4, 0.1, centers, dims, eps, 1.0)
    assert itf.n == m.n
    assert np.array_equal(itf.points, m.pts)
    assert np.array_equal(itf.normals, m.nrm)
    assert np.array_equal(itf.weights, m.w)
    assert np.array_equal(itf.eps_in, m.eps_in)


@pytest.mark.parametrize("up_tol,correct_edges", [(1e-9, True), (1e-6, False)])
def test_neighbor_list_matches_oracle(bie, orc, up_tol, correct_edges):
    itf = bie.single_dielectric_box3d(*CFG1)
    m = orc.Mesh.single_box(*CFG1)
    ups, adp = bie.build_neighbor_list(itf, 8, up_tol, correct_edges=correct_edges)
    ups_o, adp_o = orc.build_neighbor_list(m, 8, up_tol, correct_edges)
    assert ups == ups_o
    assert sorted(adp) == sorted(adp_o)


def test_correction_blocks_match_oracle(bie, orc):
    itf = bie.single_dielectric_box3d(*CFG1)
    m = orc.Mesh.single_box(*CFG1)
    C_lib = bie.laplace3d_DT_corrections(itf, max_order=8, up_tol=1e-9, correct_edges=True).tocsr()
    ups, adp = orc.build_neighbor_list(m, 8, 1e-9, True)
    C_orc = orc.DT_corrections(m, ups, adp, 1e-9).tocsr()
    D = (C_lib - C_orc).toarray()
    scale = np.abs(C_orc.toarray()).max()
    assert np.abs(D).max() <= 1e-13 * scale
    # same sparsity (structural blocks of the BSR against the CSC's nonzeros)
    assert set(zip(*C_orc.nonzero())) <= set(zip(*C_lib.nonzero()))


def test_near_release_values(bie):
    """bie_near_release_values frees the host block values and keeps the structure:
    afterwards copying the values or building a geometry from the handle is refused
    with BIE_EINVAL (no device is touched)."""
    import ctypes as C
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    itf = bie.single_dielectric_box3d(*CFG1)
    nr = itf.near(8, 1e-9, True, setup_device=-1)
    assert nr.nblocks > 0
    v = np.zeros(nr.nblocks * nr.nb * nr.nb)
    assert L.bie_near_copy(nr._h, None, None, _abi.dptr(v), None, None, None, None, None) == _abi.BIE_OK
    assert np.count_nonzero(v) > 0
    assert L.bie_near_release_values(nr._h) == _abi.BIE_OK
    assert L.bie_near_release_values(nr._h) == _abi.BIE_OK  # idempotent
    assert L.bie_near_copy(nr._h, None, None, _abi.dptr(v), None, None, None, None, None) == _abi.BIE_EINVAL
    assert "released" in _abi.last_error()
    rp = np.zeros(itf.npanels + 1, dtype=np.int32)
    assert L.bie_near_copy(nr._h, _abi.i32ptr(rp), None, None, None, None, None, None, None) == _abi.BIE_OK
    assert np.array_equal(rp, nr.rowptr)
    g = C.c_void_p()
    assert L.bie_geom_create_from_mesh(itf._h, nr._h, 0, C.byref(g)) == _abi.BIE_EINVAL
    assert not g.value
