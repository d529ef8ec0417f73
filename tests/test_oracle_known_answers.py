"""Pins the CPU oracle against the reference's own known-answer tests.

The reference (Julia) cannot run here; these restate its test assertions on the
oracle (each test cites the reference test it mirrors). No golden sigma vectors
exist in the reference, so sigma itself is pinned through invariants
(Gauss flux, total polarisation charge, residuals) and exact-assembly checks.
"""
import numpy as np
import pytest
import scipy.linalg as sla

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def sq(z, lo=-0.5, hi=0.5):
    return [[lo, lo, z], [hi, lo, z], [hi, hi, z], [lo, hi, z]]


def small(x0, y0, z, s=0.02):
    return [[x0, y0, z], [x0 + s, y0, z], [x0 + s, y0 + s, z], [x0, y0 + s, z]]


def test_best_grid(orc):
    """test/utils/best_grid.jl"""
    assert orc.best_grid_mn(20.0, 1.0, np.sqrt(2)) == (15, 1)
    assert orc.best_grid_mn(2.0, 1.0, np.sqrt(2)) == (2, 1)
    assert orc.best_grid_mn(1.0, 2.0, np.sqrt(2)) == (1, 2)
    assert orc.best_grid_mn(1.0, 1.0, 1.0) == (1, 1)
    assert orc.best_grid_mn(3.0, 2.0, 1.0) == (3, 2)
    for W, H, a in [(0.0, 1.0, 1.0), (1.0, 0.0, 1.0), (1.0, 1.0, 0.99)]:
        with pytest.raises(ValueError):
            orc.best_grid_mn(W, H, a)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 8, 12, 24, 48])
def test_gausslegendre(orc, n):
    """FastGaussQuadrature.gausslegendre: exact for polynomials of degree 2n-1, symmetric."""
    x, w = orc.gausslegendre(n)
    assert np.all(np.diff(x) > 0)
    assert np.allclose(x, -x[::-1], atol=1e-15, rtol=0)
    ref_x, ref_w = np.polynomial.legendre.leggauss(n)
    assert np.max(np.abs(x - ref_x)) < 4e-16 and np.max(np.abs(w - ref_w) / ref_w) < 2e-12
    for d in range(2 * n):
        exact = 0.0 if d % 2 else 2.0 / (d + 1)
        assert abs(np.dot(w, x ** d) - exact) < 1e-13


def test_box_geometry_and_counts(orc):
    """Config node counts and the face/normal layout (test/shape/box3d.jl:55-61)."""
    assert orc.Mesh.single_box(*CFG1).n == 2560
    m = orc.Mesh.single_box(1.0, 2.0, 3.0, 2, 10.0, 2.0, 1.0)
    assert np.array_equal(m.normals[0], [0, 0, 1]) and np.array_equal(m.normals[m.npanels - 1], [0, -1, 0])
    assert orc.Mesh.single_box(1.5, 1.0, 0.8, 6, 0.08, 4.0, 1.0).n == 42048
    assert orc.Mesh.single_box(2.0, 1.0, 1.0, 6, 0.05, 10.0, 1.0).n == 94752
    # total area of a box surface
    m = orc.Mesh.single_box(1.2, 0.8, 0.6, 6, 0.3, 2.0, 1.0)
    assert abs(m.w.sum() - 2 * (1.2 * 0.8 + 1.2 * 0.6 + 0.8 * 0.6)) < 1e-13


def test_gauss_flux_convergence(orc):
    """test/kernel/laplace3d.jl:120-137: sum_i w_i dG/dn(s, x_i) -> 1, < 1e-8 at n_quad = 6."""
    errs = []
    for nq in (2, 4, 6):
        m = orc.Mesh.single_box(1.0, 1.0, 1.0, nq, 0.3, 2.0, 1.0)
        flux = sum(orc.grad([0.1, 0.1, 0.1], m.pts[i], m.nrm[i]) * m.w[i] for i in range(m.n))
        errs.append(abs(flux - 1.0))
    assert errs[1] <= errs[0] and errs[2] <= errs[1] and errs[2] < 1e-8


def test_D_constant_density(orc):
    """test/kernel/laplace3d.jl:39-46: D 1 ~ 1/2 in the weighted mean."""
    m = orc.Mesh.single_box(1.2, 0.8, 0.6, 4, 0.2, 2.0, 1.0)
    D = m.DT_dense().T  # D[j, i] = DT[i, j] w_i / w_j ... assembled from the same kernel
    # D (src/kernel/laplace3d.jl:42-52): D[j,i] = grad(y_j, x_i, n_i) w_i
    Dm = np.zeros((m.n, m.n))
    for i in range(0, m.n, 1):
        d = m.pts[i] - m.pts
        r = np.linalg.norm(d, axis=1)
        r[i] = 1.0
        g = (d @ m.nrm[i]) / r ** 3 / (4 * np.pi) * m.w[i]
        g[i] = 0.0
        Dm[:, i] = g
    vals = Dm @ np.ones(m.n)
    assert np.dot(np.abs(vals - 0.5), m.w) < 1e-1
    del D


def test_dense_lu_solve_cfg1(orc):
    """test/solver/dielectric_box3d.jl:8-31 on the config-1 geometry (eps_box = 4)."""
    m = orc.Mesh.single_box(*CFG1)
    A = m.DT_dense(with_diag=True)
    b = orc.rhs_point(m.pts, m.nrm, [0.1, 0.1, 0.1], 1.0, 4.0)
    x = sla.lu_solve(sla.lu_factor(A), b)
    assert np.linalg.norm(A @ x - b) < 1e-10
    assert abs(np.dot(m.w, x) + 1 / 4.0 - 1.0) < 1e-1
    # matrix-free operator == dense (lhs * x_trial vs fmm3d operator < 1e-8)
    xt = np.random.default_rng(0).standard_normal(m.n)
    assert np.linalg.norm(A @ xt - orc.op_apply(m, xt)) < 1e-11
    xg, it, res = orc.gmres(m, b, None, atol=1e-12, rtol=1e-12, itmax=500)
    assert np.linalg.norm(A @ xg - b) < 1e-10
    assert abs(np.dot(m.w, xg) + 1 / 4.0 - 1.0) < 1e-1


def test_DT_panel_vs_loop(orc):
    """test/kernel/laplace3d_near.jl:66-109."""
    m = orc.Mesh.from_panels(5, [[[-0.4, -0.2, 0.1], [0.6, -0.2, 0.1], [0.6, 0.8, 0.1], [-0.4, 0.8, 0.1]],
                                 [[-0.6, -0.4, 0.7], [0.7, -0.4, 0.7], [0.7, 0.9, 0.7], [-0.6, 0.9, 0.7]]],
                             [[0, 0, 1], [0, 0, 1]])
    K = orc.DT_panel(m, 0, 1)
    nq2 = 25
    rho = 0.3 + m.pts[:nq2, 0] - 0.5 * m.pts[:nq2, 1] + 0.2 * m.pts[:nq2, 2]
    direct = np.array([sum(orc.grad(m.pts[i], m.pts[nq2 + j], m.nrm[nq2 + j]) * m.w[i] * rho[i] for i in range(nq2))
                       for j in range(nq2)])
    assert np.max(np.abs(K @ rho - direct)) < 1e-12


def test_neighbor_list_bernstein(orc):
    """test/kernel/laplace3d_near.jl:112-179."""
    m = orc.Mesh.from_panels(2, [sq(0.0), sq(0.2), small(1.0, 1.0, 1.0), small(1.0, 1.0, 1.2)], [[0, 0, 1]] * 4)
    ups, adp = orc.build_neighbor_list(m, 12, 1e-3, True)
    atol, mo = 1e-3, 12
    rho_star = atol ** (-1 / (2 * 2))
    r12 = min(orc.bernstein_rho_panel(m.corners[0], m.normals[0], p) for p in m.pts[4:8])
    r21 = min(orc.bernstein_rho_panel(m.corners[1], m.normals[1], p) for p in m.pts[0:4])
    p12 = int(np.clip(np.ceil(-np.log(atol) / (2 * np.log(r12))), 2, mo))
    p21 = int(np.clip(np.ceil(-np.log(atol) / (2 * np.log(r21))), 2, mo))
    assert r12 <= rho_star and r21 <= rho_star and p12 > 2 and p21 > 2
    assert ups[(0, 1)] == p12 and ups[(1, 0)] == p21
    assert (2, 3) not in ups and (3, 2) not in ups


def test_neighbor_list_correct_edges_flag(orc):
    """test/kernel/laplace3d_near.jl:181-226."""
    m = orc.Mesh.from_panels(2, [sq(0.0), sq(0.2)], [[0, 0, 1]] * 2, is_edge=[1, 1])
    ups, adp = orc.build_neighbor_list(m, 12, 1e-3, False)
    assert not ups and not adp
    ups, adp = orc.build_neighbor_list(m, 12, 1e-3, True)
    assert set(k for p in list(ups) + adp for k in p)


def test_neighbor_list_same_surface_skip(orc):
    """test/kernel/laplace3d_near.jl:228-256."""
    p1 = [[-0.5, -0.5, 0], [0, -0.5, 0], [0, 0, 0], [-0.5, 0, 0]]
    p2 = [[0.1, 0.1, 0], [0.6, 0.1, 0], [0.6, 0.6, 0], [0.1, 0.6, 0]]
    m = orc.Mesh.from_panels(2, [p1, p2], [[0, 0, 1]] * 2)
    ups, adp = orc.build_neighbor_list(m, 12, 1e-3, True)
    assert not ups and not adp


def test_corrections_equal_explicit_blocks(orc):
    """test/kernel/laplace3d_near.jl:290-370."""
    m = orc.Mesh.from_panels(2, [sq(0.0), sq(0.2), small(10.0, 10.0, 1.0), small(10.0, 10.0, 1.2)], [[0, 0, 1]] * 4)
    ups, adp = orc.build_neighbor_list(m, 12, 1e-3, True)
    assert set(ups) == {(0, 1), (1, 0)}
    Cm = orc.DT_corrections(m, ups, adp, 1e-3)
    rho = np.sin(0.1 * np.arange(1, m.n + 1))
    exp = np.zeros(m.n)
    b12 = orc.DT_panel_upsampled(m, 0, 1, ups[(0, 1)]) - orc.DT_panel(m, 0, 1)
    b21 = orc.DT_panel_upsampled(m, 1, 0, ups[(1, 0)]) - orc.DT_panel(m, 1, 0)
    exp[4:8] += b12 @ rho[0:4]
    exp[0:4] += b21 @ rho[4:8]
    got = Cm @ rho
    assert np.max(np.abs(got - exp)) < 1e-12
    assert np.max(np.abs(got[8:])) == 0.0


def test_upsampled_same_order_is_direct(orc):
    """test/kernel/laplace3d_near.jl:372-401: n_up == n_quad gives the direct block."""
    m = orc.Mesh.from_panels(3, [sq(0.0), sq(0.3)], [[0, 0, 1]] * 2)
    assert np.max(np.abs(orc.DT_panel_upsampled(m, 0, 1, 3) - orc.DT_panel(m, 0, 1))) < 1e-12


def test_corrected_equals_base_plus_corrections(orc):
    """test/kernel/laplace3d_near.jl:403-465 (direct sum in place of the FMM)."""
    m = orc.Mesh.from_panels(2, [sq(0.0), sq(0.2), small(1.0, 1.0, 1.0), small(1.0, 1.0, 1.2)], [[0, 0, 1]] * 4)
    ups, adp = orc.build_neighbor_list(m, 12, 1e-12, True)
    Cm = orc.DT_corrections(m, ups, adp, 1e-12)
    rho = np.cos(0.2 * np.arange(1, m.n + 1))
    base = orc.DT_apply(m.pts, m.nrm, m.w, rho)
    got = orc.op_apply(m, rho, Cm) - m.diag() * rho
    assert np.max(np.abs(got - (base + Cm @ rho))) < 1e-10


def test_upsampled_block_accuracy(orc):
    """test/kernel/laplace3d_near.jl:7-64 (upsampled D^T vs an n = 48 reference rule)."""
    ref = orc.Mesh.from_panels(48, [sq(0.0), [[-0.6, -0.6, 0.4], [0.6, -0.6, 0.4], [0.6, 0.6, 0.4], [-0.6, 0.6, 0.4]]],
                               [[0, 0, 1]] * 2)
    m = orc.Mesh.from_panels(6, ref.corners, ref.normals)
    n_ref2 = 48 * 48
    rho_ref = np.exp(-0.5 * np.sum(ref.pts[:n_ref2] ** 2, axis=1))
    # reference value at the first target node of the 6-point target panel
    tgt = m.pts[36]
    ref_val = sum(orc.grad(ref.pts[i], tgt, [0, 0, 1]) * ref.w[i] * rho_ref[i] for i in range(n_ref2))
    rho_src = np.exp(-0.5 * np.sum(m.pts[:36] ** 2, axis=1))
    up = orc.DT_panel_upsampled(m, 0, 1, 24)
    assert abs((up @ rho_src)[0] - ref_val) < 40 * 1e-8


def test_adaptive_moments_vs_cubature(orc):
    """test/kernel/laplace3d_near_adaptive.jl:21-59 (HCubature replaced by a 64-point tensor
    Gauss rule; the target is 0.3 above the panel, so the integrand is smooth)."""
    m = orc.Mesh.from_panels(4, [sq(0.0)], [[0, 0, 1]])
    pt, nt = np.array([0.1, 0.2, 0.3]), np.array([0.0, 0.0, 1.0])
    K, hit = orc.adaptive_panel_moments(m, 0, pt, nt, 1e-10, 1e-12, 4, 12)
    assert not hit
    x4, w4 = orc.gausslegendre(4)
    lam = np.array([(1 if (3 - i) % 2 == 0 else -1) * np.sqrt((1 - x4[i] ** 2) * w4[i] / 2) for i in range(4)])
    lam /= np.abs(lam).max()

    def row(u):
        t = lam / (u - x4)
        return t / t.sum()
    xg, wg = np.polynomial.legendre.leggauss(64)
    Kref = np.zeros(16)
    for a, wa in zip(xg, wg):
        ra = row(a)
        for b, wb in zip(xg, wg):
            rb = row(b)
            y = np.array([0.5 * a, 0.5 * b, 0.0])
            kv = orc.grad(y, pt, nt) * 0.25
            Kref += wa * wb * kv * np.outer(ra, rb).ravel()
    assert np.allclose(K, Kref, atol=1e-7, rtol=1e-7)


def test_touching_pair_regression(orc):
    """test/kernel/laplace3d_near_touching.jl:12-86: the adaptive (correct_edges) correction
    beats the uncorrected rule near a shared edge, and is accurate to 1e-5."""
    pa = [[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.5, 0.5, 0.0], [-0.5, 0.5, 0.0]]
    pb = [[0.5, -0.5, 0.0], [0.5, 0.5, 0.0], [0.5, 0.5, 1.0], [0.5, -0.5, 1.0]]
    m = orc.Mesh.from_panels(8, [pa, pb], [[0, 0, 1], [1, 0, 0]], eps_in=[1.0, 1.0], eps_out=[1.0, 1.0])
    sig = np.exp(-2.0 * np.sum(m.pts ** 2, axis=1))
    t = 64  # first node of panel b
    tgt, tn = m.pts[t], np.array([1.0, 0.0, 0.0])

    def quad(corners, n_ref=400):
        a, b, c, d = (np.array(v) for v in corners)
        cc, bma, dma = (a + b + c + d) / 4, b - a, d - a
        s = np.linalg.norm(bma) * np.linalg.norm(dma) / 4
        # graded Gauss rule on [-1,1]^2 (tensor of Gauss-Legendre on dyadic intervals)
        xs, ws = [], []
        g, gw = np.polynomial.legendre.leggauss(20)
        edges = np.concatenate([-1 + 2.0 ** -np.arange(30, 0, -1), [0.0], 1 - 2.0 ** -np.arange(1, 31)])
        edges = np.unique(np.concatenate([[-1.0], edges, [1.0]]))
        for lo, hi in zip(edges[:-1], edges[1:]):
            xs.append((hi - lo) / 2 * g + (hi + lo) / 2)
            ws.append((hi - lo) / 2 * gw)
        xs, ws = np.concatenate(xs), np.concatenate(ws)
        U, V = np.meshgrid(xs, xs, indexing="ij")
        W = np.outer(ws, ws)
        Y = cc + bma * (U[..., None] / 2) + dma * (V[..., None] / 2)
        D = tgt - Y
        r = np.linalg.norm(D, axis=-1)
        with np.errstate(divide="ignore", invalid="ignore"):
            k = (D @ tn) / r ** 3 / (4 * np.pi)
        k[~np.isfinite(k)] = 0.0
        return np.sum(W * k * np.exp(-2.0 * np.sum(Y ** 2, axis=-1))) * s
    ref = quad(pa) + quad(pb)
    base = orc.DT_apply(m.pts, m.nrm, m.w, sig)[t]
    u_off, a_off = orc.build_neighbor_list(m, 24, 1e-8, False)
    u_on, a_on = orc.build_neighbor_list(m, 24, 1e-8, True)
    assert a_on  # the shared edge makes a touching (adaptive) pair
    c_off = orc.DT_corrections(m, u_off, a_off, 1e-8)
    c_on = orc.DT_corrections(m, u_on, a_on, 1e-8)
    err_off = abs(base + (c_off @ sig)[t] - ref)
    err_on = abs(base + (c_on @ sig)[t] - ref)
    assert err_on < err_off
    assert err_on < 1e-5
