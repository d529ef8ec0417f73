"""Near-accurate probe potentials on the GPU (laplace3d_pottrg_fmm3d_corrected_hcubature,
src/kernel/laplace3d_near_hcubature.jl:278-316): the device operator (prolongation,
direct sum of the refined nodes, corrections) against the host operator assembled in
numpy (1e-13), against the exact single layer of the interpolated density on the cfg1 box
for probes 1e-3 .. 3e-2 from its faces (the reference's 2e-7 bar, and well below the
uncorrected error), and, for far probes, against the plain laplace3d_pottrg."""
import numpy as np
import pytest

from probe_reference import assemble, exact_potential
from test_probe_setup import THREE_PANEL_TARGETS, three_panels

pytestmark = pytest.mark.gpu

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def test_device_operator_equals_host_operator(bie):
    itf = three_panels(bie)
    j = np.arange(1, itf.n + 1)
    S = np.stack([np.cos(0.15 * j) + 0.1 * np.sin(0.27 * j), np.sin(0.4 * j), np.ones(itf.n)], axis=1)
    op = bie.laplace3d_pottrg_fmm3d_corrected_hcubature(itf, THREE_PANEL_TARGETS, 1e-10, 1e-9, 5.0)
    got = op @ S
    for c in range(3):
        host, _, _ = assemble(op, S[:, c])
        assert rel(got[:, c], host) < 1e-13


def plate(bie):
    """6 x 6 coplanar non-edge panels of side 0.2 (n_quad = 4)."""
    ns, ws = bie.gausslegendre(4)
    pan = []
    for i in range(6):
        for j in range(6):
            x0, y0 = -0.6 + 0.2 * i, -0.6 + 0.2 * j
            pan.append(bie.rect_panel3d_discretize((x0, y0, 0.0), (x0 + 0.2, y0, 0.0), (x0 + 0.2, y0 + 0.2, 0.0),
                                                   (x0, y0 + 0.2, 0.0), ns, ws, (0.0, 0.0, 1.0)))
    return bie.DielectricInterface(pan, [4.0] * 36, [1.0] * 36)


def test_near_probes_over_a_plate(bie):
    itf = plate(bie)
    rng = np.random.default_rng(11)
    T = np.column_stack([rng.uniform(-0.3, 0.3, 6), rng.uniform(-0.3, 0.3, 6), [1e-3, 3e-3, 1e-2, 2e-2, 3e-2, 5e-3]])
    x = itf.points
    sigma = np.cos(2.0 * x[:, 0]) + x[:, 1] ** 2 - 0.5 * x[:, 0] * x[:, 1]
    op = bie.laplace3d_pottrg_fmm3d_corrected_hcubature(itf, T, 1e-10, 1e-9, 5.0)
    got = op @ sigma
    base = bie.laplace3d_pottrg(itf, T) @ sigma
    ref = np.array([exact_potential(itf, sigma, t) for t in T])
    err, err_base = np.abs(got - ref), np.abs(base - ref)
    assert op.info()["capped"] == 0
    assert np.max(err) < 2e-7, err
    assert np.all(err < 1e-3 * err_base), (err, err_base)


def test_edge_panels_are_not_corrected(bie):
    """build_target_neighbor_list(refined, targets, false): a probe beside a box corner, in
    range of edge panels only, gets its refined panels but no corrections
    (src/kernel/laplace3d_near_hcubature.jl:302)."""
    itf = bie.single_dielectric_box3d(*CFG1)
    corner = np.array([[0.6, 0.4, 0.3]]) + 2e-3
    op = bie.laplace3d_pottrg_fmm3d_corrected_hcubature(itf, corner, 1e-10, 1e-9, 5.0)
    inf = op.info()
    assert inf["npanels_refined"] > itf.npanels and inf["nnz_corrections"] == 0
    sigma = np.ones(itf.n)
    phi = op @ sigma
    host, _, _ = assemble(op, sigma)
    assert rel(phi, host) < 1e-13


def test_far_probes_match_plain_potential(bie):
    itf = bie.single_dielectric_box3d(*CFG1)
    T = np.array([[3.0, 0.1, 0.2], [-2.5, 1.0, 0.3], [0.2, 0.1, 4.0]])
    sigma = np.sin(0.01 * np.arange(itf.n))
    op = bie.laplace3d_pottrg_fmm3d_corrected_hcubature(itf, T, 1e-10, 1e-9, 5.0)
    assert op.info()["nnz_corrections"] == 0
    assert rel(op @ sigma, bie.laplace3d_pottrg(itf, T) @ sigma) < 1e-13
