"""Host set-up of near-accurate probe potentials (laplace3d_pottrg_fmm3d_corrected_hcubature,
src/kernel/laplace3d_near_hcubature.jl:278-316), checked on the CPU with the operator
(S_refined + C) P assembled in numpy from the library's host set-up. The cases are those
of the reference's tests (test/kernel/laplace3d_near.jl:636-845): corrected error below the
uncorrected one and below 2e-7 against the all-panels adaptive integral; far probes give the
uncorrected operator; target-driven refinement stops at the smallest panel size; unsplit
panels keep their density."""
import numpy as np
import pytest

from probe_reference import assemble, exact_potential, smooth_potential


def three_panels(bie):
    ns, ws = bie.gausslegendre(3)
    n = (0.0, 0.0, 1.0)
    p1 = bie.rect_panel3d_discretize((-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0), ns, ws, n)
    p2 = bie.rect_panel3d_discretize((-0.5, -0.5, 0.15), (0.5, -0.5, 0.15), (0.5, 0.5, 0.15), (-0.5, 0.5, 0.15),
                                     ns, ws, n)
    p3 = bie.rect_panel3d_discretize((1.2, 1.2, 0.8), (1.4, 1.2, 0.8), (1.4, 1.4, 0.8), (1.2, 1.4, 0.8), ns, ws, n)
    return bie.DielectricInterface([p1, p2, p3], [2.0] * 3, [1.0] * 3)


THREE_PANEL_TARGETS = np.array([[0.05, 0.04, 0.01], [-0.10, 0.06, 0.18], [0.30, -0.20, 0.55]])


def two_panels(bie, far_corner):
    ns, ws = bie.gausslegendre(2)
    n = (0.0, 0.0, 1.0)
    p1 = bie.rect_panel3d_discretize((-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0), ns, ws, n)
    x0, x1 = far_corner
    p2 = bie.rect_panel3d_discretize((x0, x0, 0.0), (x1, x0, 0.0), (x1, x1, 0.0), (x0, x1, 0.0), ns, ws, n)
    return bie.DielectricInterface([p1, p2], [2.0] * 2, [1.0] * 2)


def test_corrected_beats_smooth_quadrature(bie):
    itf = three_panels(bie)
    j = np.arange(1, itf.n + 1)
    sigma = np.cos(0.15 * j) + 0.1 * np.sin(0.27 * j)
    op = bie.ProbePotentialOperator(itf, THREE_PANEL_TARGETS, 1e-9, 5.0, device=-1)
    got, _, _ = assemble(op, sigma)
    ref = np.array([exact_potential(itf, sigma, t) for t in THREE_PANEL_TARGETS])
    base = smooth_potential(itf.points, itf.weights, sigma, THREE_PANEL_TARGETS)
    err_base, err = np.max(np.abs(base - ref)), np.max(np.abs(got - ref))
    assert err < err_base
    assert err < 2e-7
    inf = op.info()
    assert inf["capped"] == 0 and inf["ncubatures"] > 0 and inf["nnz_corrections"] > 0
    # the remaining error is the smooth quadrature of panels just outside the correction
    # radius; with a wider radius the corrected operator reaches the cubature accuracy
    wide, _, _ = assemble(bie.ProbePotentialOperator(itf, THREE_PANEL_TARGETS, 1e-9, 20.0, device=-1), sigma)
    assert np.max(np.abs(wide - ref)) < 1e-10


def test_far_probes_give_the_smooth_operator(bie):
    ns, ws = bie.gausslegendre(2)
    n = (0.0, 0.0, 1.0)
    p1 = bie.rect_panel3d_discretize((-0.5, -0.5, 0.0), (0.5, -0.5, 0.0), (0.5, 0.5, 0.0), (-0.5, 0.5, 0.0), ns, ws, n)
    p2 = bie.rect_panel3d_discretize((-0.5, -0.5, 0.2), (0.5, -0.5, 0.2), (0.5, 0.5, 0.2), (-0.5, 0.5, 0.2),
                                     ns, ws, n)
    itf = bie.DielectricInterface([p1, p2], [2.0] * 2, [1.0] * 2)
    T = np.array([[3.0, 3.0, 3.0], [3.5, 3.5, 3.5]])
    op = bie.ProbePotentialOperator(itf, T, 1e-8, 0.1, device=-1)
    inf = op.info()
    assert inf["nnz_corrections"] == 0 and inf["npanels_refined"] == itf.npanels
    sigma = np.sin(0.3 * np.arange(1, itf.n + 1))
    got, _, _ = assemble(op, sigma)
    assert np.max(np.abs(got - smooth_potential(itf.points, itf.weights, sigma, T))) < 1e-12


def test_target_driven_refinement(bie):
    itf = two_panels(bie, (2.0, 2.4))
    op = bie.ProbePotentialOperator(itf, np.array([[0.02, -0.01, 0.03]]), 1e-9, 5.0, device=-1)
    R = op.refinement()
    assert len(R["parent"]) > itf.npanels
    assert np.any(R["parent"] == 0) and np.any(R["from_split"])
    c = itf.corners
    min_len = min(max(np.linalg.norm(c[p, 0] - c[p, 1]), np.linalg.norm(c[p, 1] - c[p, 2])) for p in range(itf.npanels))
    rc = R["corners"]
    lens = np.maximum(np.linalg.norm(rc[:, 0] - rc[:, 1], axis=1), np.linalg.norm(rc[:, 1] - rc[:, 2], axis=1))
    assert np.all(lens <= min_len + 1e-14)


def test_prolongation_keeps_unsplit_panels_and_interpolates(bie):
    itf = two_panels(bie, (5.0, 6.0))
    op = bie.ProbePotentialOperator(itf, np.array([[0.01, -0.02, 0.03]]), 1e-9, 5.0, device=-1)
    sigma = np.sin(0.17 * np.arange(1, itf.n + 1))
    _, s_ref, R = assemble(op, sigma)
    q2 = itf.n_quad ** 2
    for r, (par, split) in enumerate(zip(R["parent"], R["from_split"])):
        if not split:
            assert np.array_equal(s_ref[r * q2:(r + 1) * q2], sigma[par * q2:(par + 1) * q2])
    # a density linear in the coordinates is interpolated exactly onto the refined nodes
    lin = 0.3 + 1.7 * itf.points[:, 0] - 0.4 * itf.points[:, 1]
    _, s_lin, R = assemble(op, lin)
    expect = 0.3 + 1.7 * R["points"][:, 0] - 0.4 * R["points"][:, 1]
    assert np.max(np.abs(s_lin - expect)) < 1e-13
    # partition of unity: every prolongation row sums to one
    rows = np.add.reduceat(R["pval"], R["prow"][:-1])
    assert np.max(np.abs(rows - 1.0)) < 1e-14
