"""Correction blocks computed on the GPU equal the host's bitwise: the adaptive
(touching-pair) moment sums (src/kernel/laplace3d_near_adaptive.jl:308-387) and the
upsampled blocks (src/kernel/laplace3d_near_upsampling.jl:127-270: Mt K_up - K_direct per
near pair, one upsampling order per source panel). Both kernels follow the host's
operation order with explicitly rounded arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", [(1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0), (1.5, 1.0, 0.8, 6, 0.08, 4.0, 1.0)])
def test_adaptive_blocks_gpu_bitwise_equal_host(bie, cfg):
    itf = bie.single_dielectric_box3d(*cfg)
    host = itf.near(8, 1e-9, True, setup_device=-1)
    itf2 = bie.single_dielectric_box3d(*cfg)
    dev = itf2.near(8, 1e-9, True, setup_device=0)
    assert len(dev.adaptive) > 0 and len(dev.upsample) > 0
    assert np.array_equal(host.rowptr, dev.rowptr)
    assert np.array_equal(host.col, dev.col)
    assert np.array_equal(host.val, dev.val)


def test_adaptive_blocks_gpu_multibox(bie):
    boxes = [{"center": (-0.45, 0.0, 0.0), "Lx": 0.6, "Ly": 0.5, "Lz": 0.4},
             {"center": (0.45, 0.05, 0.0), "Lx": 0.5, "Ly": 0.6, "Lz": 0.5}]
    a = bie.multi_dielectric_box3d(6, 0.12, boxes, [4.0, 12.0], 1.0).near(8, 1e-9, True, setup_device=-1)
    b = bie.multi_dielectric_box3d(6, 0.12, boxes, [4.0, 12.0], 1.0).near(8, 1e-9, True, setup_device=0)
    assert np.array_equal(a.val, b.val)


def test_released_host_blocks_read_back_from_device(bie):
    """keep_host_blocks=False: the host copy of the blocks is freed once the geometry is
    on the device; the values read back from the device equal the host build bitwise, and
    solves agree to rounding."""
    cfg = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)
    a, b = bie.single_dielectric_box3d(*cfg), bie.single_dielectric_box3d(*cfg)
    op_a = bie.lhs_dielectric_box3d_fmm3d_corrected(a, 1e-12, 1e-9, 8)
    op_b = bie.lhs_dielectric_box3d_fmm3d_corrected(b, 1e-12, 1e-9, 8, keep_host_blocks=False)
    assert not op_a.near.released and op_b.near.released
    assert np.array_equal(op_b.near.val, op_a.near.val)
    F = bie.rhs_dielectric_box3d(a, bie.PointSource((0.1, 0.1, 0.1), 1.0), 4.0)
    Sa, _ = bie.gpu_solve(op_a, F, rtol=1e-12)
    Sb, _ = bie.gpu_solve(op_b, F, rtol=1e-12)
    # (each handle tunes its own launch shapes, so the rounding may differ)
    assert np.linalg.norm(Sa - Sb) <= 1e-13 * np.linalg.norm(Sa)
    with pytest.raises(RuntimeError):
        b.geom(op_b.near, device=1)
