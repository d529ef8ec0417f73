"""Adaptive (touching-pair) correction blocks computed on the GPU equal the host's
bitwise: the kernel follows the host's operation order with explicitly rounded
arithmetic (src/kernel/laplace3d_near_adaptive.jl:308-387 is the reference sum)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg", [(1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0), (1.5, 1.0, 0.8, 6, 0.08, 4.0, 1.0)])
def test_adaptive_blocks_gpu_bitwise_equal_host(bie, cfg):
    itf = bie.single_dielectric_box3d(*cfg)
    host = itf.near(8, 1e-9, True, setup_device=-1)
    itf2 = bie.single_dielectric_box3d(*cfg)
    dev = itf2.near(8, 1e-9, True, setup_device=0)
    assert len(dev.adaptive) > 0
    assert np.array_equal(host.rowptr, dev.rowptr)
    assert np.array_equal(host.col, dev.col)
    assert np.array_equal(host.val, dev.val)


def test_adaptive_blocks_gpu_multibox(bie):
    boxes = [{"center": (-0.45, 0.0, 0.0), "Lx": 0.6, "Ly": 0.5, "Lz": 0.4},
             {"center": (0.45, 0.05, 0.0), "Lx": 0.5, "Ly": 0.6, "Lz": 0.5}]
    a = bie.multi_dielectric_box3d(6, 0.12, boxes, [4.0, 12.0], 1.0).near(8, 1e-9, True, setup_device=-1)
    b = bie.multi_dielectric_box3d(6, 0.12, boxes, [4.0, 12.0], 1.0).near(8, 1e-9, True, setup_device=0)
    assert np.array_equal(a.val, b.val)
