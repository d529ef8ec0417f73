"""Generates the oracle's sigma columns on the two large single-box configurations
(seeded, deterministic; takes a few minutes on 8 host cores).

    python tests/golden/make_large.py [cfg3] [cfg2]

The reference ships no sigma vectors, so these columns come from the CPU oracle
(oracle/bie_oracle.c), which restates the reference's corrected operator
(src/kernel/laplace3d_near.jl:395-419, src/solver/dielectric_box3d.jl:48-92) with the
FMM replaced by the exact direct sum, and solves it with unrestarted GMRES (MGS +
Givens) to rtol 1e-13, followed by one step of iterative refinement in FP64 (the true
residual r = f - A x is solved for to rtol 1e-3 and the correction added), which takes
the true residual, recomputed afterwards and stored, to the FP64 floor:

  cfg3_sigma.npz  box 1.5 x 1.0 x 0.8, n_quad 6, l_ec 0.08, eps_in 4, eps_out 1
                  (N = 42,048); 4 point sources uniform in the inner 90 % of the box,
                  charges ~ N(0, 1) (seed 3: the first four columns of the benchmark's
                  first 64-source batch), eps_src 4
  cfg2_sigma.npz  box 2.0 x 1.0 x 1.0, n_quad 6, l_ec 0.05, eps_in 10, eps_out 1
                  (N = 94,752); 1 point source uniform in the inner 80 %, charge +-1
                  (seed 2: the first column of the benchmark's first 8-source batch)

Both use the near-field corrections at up_tol 1e-9, max_order 8, correct_edges.
Each file holds the sources, sigma (N x k, column-major), the oracle's true
relative residual ||f - A sigma|| / ||f|| per column and mesh fingerprints.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

CASES = {
    "cfg3": dict(box=(1.5, 1.0, 0.8), nq=6, l_ec=0.08, eps_in=4.0, seed=3, batch=64, take=4, inner=0.9,
                 charges="normal", rtol=1e-13),
    "cfg2": dict(box=(2.0, 1.0, 1.0), nq=6, l_ec=0.05, eps_in=10.0, seed=2, batch=8, take=1, inner=0.8,
                 charges="pm1", rtol=1e-13),
}


def sources(c):
    """The first `take` sources of the seeded batch (positions drawn first, then charges)."""
    rng = np.random.default_rng(c["seed"])
    half = np.array(c["box"]) / 2 * c["inner"]
    pos = rng.uniform(-half, half, size=(c["batch"], 3))
    q = rng.standard_normal(c["batch"]) if c["charges"] == "normal" else rng.choice([-1.0, 1.0], size=c["batch"])
    return pos[: c["take"]], q[: c["take"]]


def make(name):
    c = CASES[name]
    t0 = time.perf_counter()
    m = oracle.Mesh.single_box(*c["box"], c["nq"], c["l_ec"], c["eps_in"], 1.0)
    ups, adp = oracle.build_neighbor_list(m, 8, 1e-9, True)
    Cm = oracle.DT_corrections(m, ups, adp, 1e-9)
    print(f"{name}: N={m.n}, {len(ups)} upsampled + {len(adp)} adaptive pairs, nnz={Cm.nnz}, "
          f"set-up {time.perf_counter() - t0:.1f} s", flush=True)
    pos, q = sources(c)
    sig, res, its = [], [], []
    for s, qq in zip(pos, q):
        f = oracle.rhs_point(m.pts, m.nrm, s, qq, c["eps_in"])
        t1 = time.perf_counter()
        x, it, _ = oracle.gmres(m, f, Cm, atol=0.0, rtol=c["rtol"], itmax=600)
        resid = f - oracle.op_apply(m, x, Cm)
        d, it2, _ = oracle.gmres(m, resid, Cm, atol=0.0, rtol=1e-3, itmax=100)
        x = x + d
        it += it2
        r = np.linalg.norm(f - oracle.op_apply(m, x, Cm)) / np.linalg.norm(f)
        print(f"  column {len(sig)}: {it} iterations, true rel residual {r:.2e}, {time.perf_counter() - t1:.1f} s",
              flush=True)
        sig.append(x)
        res.append(r)
        its.append(it)
    np.savez_compressed(
        os.path.join(HERE, f"{name}_sigma.npz"),
        n=m.n, npanels=m.npanels, points_sum=m.pts.sum(axis=0), weights_sum=m.w.sum(),
        correction_nnz=Cm.nnz, src=pos, q=q, eps_src=c["eps_in"],
        sigma=np.asfortranarray(np.stack(sig, axis=1)), true_rel_resid=np.array(res),
        iterations=np.array(its), rtol=c["rtol"])
    print("wrote", os.path.join(HERE, f"{name}_sigma.npz"), flush=True)


def main():
    names = [a for a in sys.argv[1:] if a in CASES] or list(CASES)
    oracle.build()
    for name in names:
        make(name)


if __name__ == "__main__":
    main()
