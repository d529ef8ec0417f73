"""Test-side references for near-accurate probe potentials (numpy).

``interp_potential`` integrates a panel's interpolated density against the Laplace
single-layer kernel by Gauss-Legendre quadrature on a quadtree of parameter cells refined
towards the probe (a cell is split while its size exceeds a quarter of its distance to the
probe), the quantity laplace3d_pottrg_near computes per panel with adaptive cubature
(src/kernel/laplace3d_near.jl:447-508). ``assemble`` applies the host operator
(S_refined + C) P of a ProbePotentialOperator with numpy."""
import numpy as np

FOUR_PI = 4.0 * np.pi


def bary_rows(x, lam, q):
    """Barycentric Lagrange rows at the points q (no q on a node)."""
    d = q[:, None] - x[None, :]
    r = lam[None, :] / d
    return r / r.sum(axis=1, keepdims=True)


def interp_potential(corners, glx, bary, sig_panel, t, n_gl=10, max_depth=40):
    a, b, c, d = (np.asarray(v, dtype=float) for v in corners)
    cc = (a + b + c + d) / 4
    bma, dma = b - a, d - a
    scale = np.linalg.norm(bma) * np.linalg.norm(dma) / 4
    L = max(np.linalg.norm(bma), np.linalg.norm(dma))
    nq = len(glx)
    S = np.asarray(sig_panel, dtype=float).reshape(nq, nq)
    leaves = []
    stack = [(-1.0, 1.0, -1.0, 1.0, 0)]
    while stack:
        u0, u1, v0, v1, depth = stack.pop()
        uc, vc = (u0 + u1) / 2, (v0 + v1) / 2
        p = cc + bma * uc / 2 + dma * vc / 2
        size = L * max(u1 - u0, v1 - v0) / 2
        dist = np.linalg.norm(p - t) - size
        if depth < max_depth and size > 0.25 * max(dist, 1e-300):
            stack += [(u0, uc, v0, vc, depth + 1), (uc, u1, v0, vc, depth + 1),
                      (u0, uc, vc, v1, depth + 1), (uc, u1, vc, v1, depth + 1)]
        else:
            leaves.append((u0, u1, v0, v1))
    gx, gw = np.polynomial.legendre.leggauss(n_gl)
    lv = np.array(leaves)
    hu, hv = (lv[:, 1] - lv[:, 0]) / 2, (lv[:, 3] - lv[:, 2]) / 2
    U = ((lv[:, 0] + lv[:, 1]) / 2)[:, None] + hu[:, None] * gx[None, :]   # leaves x n_gl
    V = ((lv[:, 2] + lv[:, 3]) / 2)[:, None] + hv[:, None] * gx[None, :]
    uu = np.repeat(U, n_gl, axis=1).ravel()          # (leaf, i, j) -> u_i
    vv = np.tile(V, (1, n_gl)).ravel()               # (leaf, i, j) -> v_j
    ww = (hu * hv)[:, None] * np.outer(gw, gw).ravel()[None, :]
    rx, ry = bary_rows(glx, bary, uu), bary_rows(glx, bary, vv)
    sig = np.einsum("pi,ij,pj->p", rx, S, ry)
    P = cc[None, :] + np.outer(uu / 2, bma) + np.outer(vv / 2, dma)
    G = 1.0 / (FOUR_PI * np.linalg.norm(P - t[None, :], axis=1))
    return float(np.sum(ww.ravel() * sig * G) * scale)


def exact_potential(itf, sigma, t):
    """Sum over every panel of its interpolated density's exact potential at t."""
    glx, bary = np.asarray(itf.panels[0].gl_xs), np.asarray(itf.panels[0].bary_weights)
    q2 = itf.n_quad ** 2
    return sum(interp_potential(itf.corners[p], glx, bary, sigma[p * q2:(p + 1) * q2], np.asarray(t))
               for p in range(itf.npanels))


def smooth_potential(points, weights, sigma, T):
    """Smooth-quadrature single layer: sum_j w_j sigma_j / (4 pi |t - y_j|)."""
    D = np.linalg.norm(T[:, None, :] - points[None, :, :], axis=2)
    return (weights[None, :] * sigma[None, :] / (FOUR_PI * D)).sum(axis=1)


def csr_apply(rowptr, col, val, x, nrows):
    y = np.zeros(nrows)
    for r in range(nrows):
        s = slice(rowptr[r], rowptr[r + 1])
        y[r] = np.dot(val[s], x[col[s]])
    return y


def assemble(op, sigma):
    """(S_refined + C) P sigma from the operator's host set-up."""
    R = op.refinement()
    nr = len(R["weights"])
    s_ref = csr_apply(R["prow"], R["pcol"], R["pval"], np.asarray(sigma, dtype=float), nr)
    M = op.T.shape[0]
    return (smooth_potential(R["points"], R["weights"], s_ref, op.T)
            + csr_apply(R["crow"], R["ccol"], R["cval"], s_ref, M)), s_ref, R


def pottrg_near(itf, sigma, t, range_factor=5.0):
    """laplace3d_pottrg_near (src/kernel/laplace3d_near.jl:447-508): panels whose centre is
    within range_factor * max(|b - a|, |d - a|) / n_quad of t are integrated exactly (here by
    the quadtree Gauss rule of interp_potential), the others by their smooth quadrature."""
    t = np.asarray(t, dtype=float)
    nq = itf.n_quad
    q2 = nq * nq
    glx, bary = np.asarray(itf.panels[0].gl_xs), np.asarray(itf.panels[0].bary_weights)
    c = itf.corners
    cc = c.mean(axis=1)
    l_panel = np.maximum(np.linalg.norm(c[:, 1] - c[:, 0], axis=1), np.linalg.norm(c[:, 3] - c[:, 0], axis=1))
    near = np.linalg.norm(cc - t[None, :], axis=1) <= range_factor * l_panel / nq
    far_nodes = np.repeat(~near, q2)
    val = float(smooth_potential(itf.points[far_nodes], itf.weights[far_nodes], sigma[far_nodes], t[None, :])[0])
    for p in np.where(near)[0]:
        val += interp_potential(c[p], glx, bary, sigma[p * q2:(p + 1) * q2], t)
    return val
