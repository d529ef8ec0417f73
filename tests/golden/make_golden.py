"""Generates the golden fixtures of tests/golden from the CPU oracle (seeded, deterministic).

    python tests/golden/make_golden.py

The reference ships no sigma vectors for this path, so the fixtures are the
oracle's dense answers on the small configuration (box 1.2 x 0.8 x 0.6, n_quad 4,
l_ec 0.2, eps_in 4, eps_out 1; N = 2560), with one PointSource at (0.1, 0.1, 0.1),
charge 1, eps_src 4:
  sigma_plain      lu(D^T + diag) \\ f            (lhs_dielectric_box3d + solve_lu)
  sigma_corrected  lu(D^T + C + diag) \\ f        (up_tol 1e-9, max_order 8, correct_edges)
  sigma_block      the same corrected system for 8 seeded sources (seed 1)
plus mesh fingerprints and the neighbour-list / correction sizes.
"""
import os
import sys

import numpy as np
import scipy.linalg as sla

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


def main():
    oracle.build()
    m = oracle.Mesh.single_box(*CFG1)
    ups, adp = oracle.build_neighbor_list(m, 8, 1e-9, True)
    Cm = oracle.DT_corrections(m, ups, adp, 1e-9)
    A = m.DT_dense(with_diag=True)
    f = oracle.rhs_point(m.pts, m.nrm, (0.1, 0.1, 0.1), 1.0, 4.0)
    lu_plain = sla.lu_factor(A)
    lu_corr = sla.lu_factor(A + Cm.toarray())
    rng = np.random.default_rng(1)
    src = rng.uniform(-0.25, 0.25, (8, 3))
    q = rng.standard_normal(8)
    F = np.stack([oracle.rhs_point(m.pts, m.nrm, s, c, 4.0) for s, c in zip(src, q)], axis=1)
    np.savez_compressed(
        os.path.join(HERE, "cfg1_sigma.npz"),
        n=m.n, npanels=m.npanels,
        points_sum=m.pts.sum(axis=0), weights_sum=m.w.sum(), weights_sq=np.dot(m.w, m.w),
        n_upsampled_pairs=len(ups), n_adaptive_pairs=len(adp), correction_nnz=Cm.nnz,
        correction_fro=np.sqrt((Cm.multiply(Cm)).sum()),
        rhs=f,
        sigma_plain=sla.lu_solve(lu_plain, f),
        sigma_corrected=sla.lu_solve(lu_corr, f),
        block_src=src, block_q=q,
        sigma_block=sla.lu_solve(lu_corr, F),
    )
    print("wrote", os.path.join(HERE, "cfg1_sigma.npz"))


if __name__ == "__main__":
    main()
