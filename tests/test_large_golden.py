"""The GPU solver against the oracle's sigma on the two large single-box configurations
(tests/golden/cfg3_sigma.npz, cfg2_sigma.npz, made by tests/golden/make_large.py: the
oracle's corrected operator, src/kernel/laplace3d_near.jl:395-419 with the exact direct
sum for the FMM, solved by unrestarted GMRES to rtol 1e-13 and one FP64 refinement step;
true relative residuals 1.1e-15 to 1.6e-15 (cfg3) and 7.0e-15 (cfg2)).

  cfg3  box 1.5 x 1.0 x 0.8, n_quad 6, l_ec 0.08, eps_in 4 (N = 42,048), 4 oracle columns
  cfg2  box 2.0 x 1.0 x 1.0, n_quad 6, l_ec 0.05, eps_in 10 (N = 94,752), 1 oracle column

Bars: plain FP64 GPU solve within 1e-12 relative in sigma per column; the refined
split-BF16 tensor-core solve (the benchmark's arithmetic, inside a block of the benchmark's
width) within 1e-8."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = {
    "cfg3": dict(box=(1.5, 1.0, 0.8), nq=6, l_ec=0.08, eps_in=4.0, block=64, half=0.9, seed=3),
    "cfg2": dict(box=(2.0, 1.0, 1.0), nq=6, l_ec=0.05, eps_in=10.0, block=8, half=0.8, seed=2),
}


def load(name):
    return dict(np.load(os.path.join(HERE, "golden", f"{name}_sigma.npz")))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fixture_matches_library_mesh(bie, name):
    """The fixture was made on the mesh the library builds (node count and fingerprints) and
    the oracle's own true residual is below 1e-14."""
    c, g = CASES[name], load(name)
    itf = bie.single_dielectric_box3d(*c["box"], c["nq"], c["l_ec"], c["eps_in"], 1.0)
    assert itf.n == g["n"] and itf.npanels == g["npanels"]
    assert np.array_equal(itf.points.sum(axis=0), g["points_sum"])
    assert itf.weights.sum() == g["weights_sum"]
    assert g["sigma"].shape == (itf.n, len(g["q"]))
    assert np.all(g["true_rel_resid"] < 1e-14)
    # total polarisation charge sum w sigma = q (1 - 1/eps_in) (test/solver/dielectric_box3d.jl:26-30)
    for col, q in enumerate(g["q"]):
        assert abs(np.dot(itf.weights, g["sigma"][:, col]) - q * (1 - 1 / c["eps_in"])) < 0.1 * abs(q)


@pytest.fixture(scope="module")
def systems(bie):
    out = {}

    def get(name):
        if name not in out:
            c, g = CASES[name], load(name)
            itf = bie.single_dielectric_box3d(*c["box"], c["nq"], c["l_ec"], c["eps_in"], 1.0)
            op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
            srcs = [bie.PointSource(tuple(p), float(q)) for p, q in zip(g["src"], g["q"])]
            out[name] = (c, g, itf, op, srcs)
        return out[name]
    return get


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_plain_fp64_vs_oracle(bie, systems, name):
    c, g, itf, op, srcs = systems(name)
    S, st = bie.gpu_solve_sources(op, srcs, float(g["eps_src"]), rtol=1e-14, itmax=600, precision="fp64")
    for col in range(len(srcs)):
        assert rel(S[:, col], g["sigma"][:, col]) < 1e-12, (name, col)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_refined_block_vs_oracle(bie, systems, name):
    """The oracle's columns first, in a block of the benchmark's width filled with further
    seeded interior sources; split-BF16 x3 tensor-core operator inside FP64 refinement to
    rtol 1e-10."""
    c, g, itf, op, srcs = systems(name)
    rng = np.random.default_rng(c["seed"] + 1000)
    half = np.array(c["box"]) / 2 * c["half"]
    extra = [bie.PointSource(tuple(rng.uniform(-half, half)), float(rng.standard_normal()))
             for _ in range(c["block"] - len(srcs))]
    S, st = bie.gpu_solve_sources(op, srcs + extra, float(g["eps_src"]), rtol=1e-10, itmax=600, precision="bf16x3")
    assert st.solved and st.lowp_matvecs > 0
    for col in range(len(srcs)):
        assert rel(S[:, col], g["sigma"][:, col]) < 1e-8, (name, col)
