"""A DielectricInterface handed over panel by panel, the way a Julia caller passes a
reference-built interface (src/core/panels.jl:5-22, 64-68: each FlatPanel's corners,
normal and is_edge, and the per-panel eps_in / eps_out) through bie_mesh_from_panels,
gives the same operator as the library's own mesher: on the small box (1.2 x 0.8 x 0.6,
n_quad 4, l_ec 0.2) the nodes, weights, diagonal and correction blocks are bit-identical
(CPU), and so is the plain FP64 GPU solution (GPU)."""
import ctypes as C

import numpy as np
import pytest

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def from_panels(bie, ref):
    """The interface rebuilt through the C ABI from the panel data alone (12 x P corners,
    3 x P normals, is_edge, eps_in, eps_out), as the Julia binding packs itf.panels."""
    from dielectricbie_jl_b200 import _abi
    P = ref.npanels
    corners = np.ascontiguousarray(ref.corners.reshape(P, 12))
    normals = np.ascontiguousarray(ref.panel_normals)
    ie = np.ascontiguousarray(ref.is_edge, dtype=np.intc)
    ei, eo = np.ascontiguousarray(ref.eps_in), np.ascontiguousarray(ref.eps_out)
    h = C.c_void_p()
    _abi.check(_abi.lib().bie_mesh_from_panels(P, ref.n_quad, _abi.dptr(corners), _abi.dptr(normals),
                                               _abi.iptr(ie), _abi.dptr(ei), _abi.dptr(eo), C.byref(h)))
    return bie.DielectricInterface(_handle=h)


def test_panel_by_panel_mesh_is_bit_identical(bie):
    ref = bie.single_dielectric_box3d(*CFG1)
    itf = from_panels(bie, ref)
    assert itf.n == ref.n == 2560 and itf.npanels == ref.npanels
    for a, b in ((itf.points, ref.points), (itf.normals, ref.normals), (itf.weights, ref.weights),
                 (itf.diag, ref.diag), (itf.corners, ref.corners), (itf.is_edge, ref.is_edge)):
        assert np.array_equal(a, b)
    # the Python FlatPanel route (DielectricInterface(panels, eps_in, eps_out)) gives the same
    itf2 = bie.DielectricInterface(ref.panels, ref.eps_in, ref.eps_out)
    assert np.array_equal(itf2.points, ref.points) and np.array_equal(itf2.weights, ref.weights)
    n1, n2 = itf.near(8, 1e-9, True, setup_device=-1), ref.near(8, 1e-9, True, setup_device=-1)
    assert n1.upsample == n2.upsample and n1.adaptive.keys() == n2.adaptive.keys()
    assert np.array_equal(n1.rowptr, n2.rowptr) and np.array_equal(n1.col, n2.col)
    assert np.array_equal(n1.val, n2.val)


@pytest.mark.gpu
def test_panel_by_panel_solve_is_bit_identical(bie, monkeypatch):
    # launch shapes fixed by the model (the autotuner's timing choice changes the summation order)
    monkeypatch.setenv("BIE_NO_AUTOTUNE", "1")
    ref = bie.single_dielectric_box3d(*CFG1)
    itf = from_panels(bie, ref)
    f = bie.rhs_dielectric_box3d(ref, bie.PointSource((0.1, 0.1, 0.1), 1.0), 4.0)
    assert np.array_equal(f, bie.rhs_dielectric_box3d(itf, bie.PointSource((0.1, 0.1, 0.1), 1.0), 4.0))
    s_ref, st_ref = bie.gpu_solve(bie.lhs_dielectric_box3d_fmm3d_corrected(ref, 1e-12, 1e-9, 8), f, rtol=1e-13)
    s, st = bie.gpu_solve(bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8), f, rtol=1e-13)
    assert st.solved and st.iterations == st_ref.iterations
    assert np.array_equal(s, s_ref)
