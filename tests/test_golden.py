"""Golden fixtures (tests/golden/cfg1_sigma.npz, made by tests/golden/make_golden.py
from the oracle): the oracle and the library's host set-up reproduce them on CPU,
and the GPU solves match them at the parity bars (plain FP64 1e-12, refined 1e-8)."""
import os

import numpy as np
import pytest
import scipy.linalg as sla

HERE = os.path.dirname(os.path.abspath(__file__))
CFG1 = (1.2, 0.8, 0.6, 4, 0.2, 4.0, 1.0)


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(HERE, "golden", "cfg1_sigma.npz")))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_oracle_reproduces_golden(orc, gold):
    m = orc.Mesh.single_box(*CFG1)
    assert m.n == gold["n"] == 2560 and m.npanels == gold["npanels"]
    assert np.array_equal(m.pts.sum(axis=0), gold["points_sum"])
    f = orc.rhs_point(m.pts, m.nrm, (0.1, 0.1, 0.1), 1.0, 4.0)
    assert np.array_equal(f, gold["rhs"])
    ups, adp = orc.build_neighbor_list(m, 8, 1e-9, True)
    assert len(ups) == gold["n_upsampled_pairs"] and len(adp) == gold["n_adaptive_pairs"]
    Cm = orc.DT_corrections(m, ups, adp, 1e-9)
    assert Cm.nnz == gold["correction_nnz"]
    A = m.DT_dense(with_diag=True)
    assert rel(sla.lu_solve(sla.lu_factor(A), f), gold["sigma_plain"]) < 1e-13
    # total polarisation charge sum w sigma = 1 - 1/eps_in (test/solver/dielectric_box3d.jl:26-30)
    assert abs(np.dot(m.w, gold["sigma_corrected"]) - (1 - 1 / 4.0)) < 0.1


def test_library_setup_reproduces_golden(bie, gold):
    itf = bie.single_dielectric_box3d(*CFG1)
    assert itf.n == gold["n"]
    assert np.array_equal(itf.points.sum(axis=0), gold["points_sum"])
    assert itf.weights.sum() == gold["weights_sum"]
    ups, adp = bie.build_neighbor_list(itf, 8, 1e-9, correct_edges=True)
    assert len(ups) == gold["n_upsampled_pairs"] and len(adp) == gold["n_adaptive_pairs"]
    C = bie.laplace3d_DT_corrections(itf, max_order=8, up_tol=1e-9, correct_edges=True)
    fro = np.sqrt((C.data ** 2).sum())
    assert abs(fro - gold["correction_fro"]) <= 1e-12 * gold["correction_fro"]


@pytest.mark.gpu
def test_gpu_solves_match_golden(bie, gold):
    itf = bie.single_dielectric_box3d(*CFG1)
    f = bie.rhs_dielectric_box3d(itf, bie.PointSource((0.1, 0.1, 0.1), 1.0), 4.0)
    assert rel(f, gold["rhs"]) < 1e-15
    op_plain = bie.lhs_dielectric_box3d(itf)
    s, st = bie.gpu_solve(op_plain, f, rtol=1e-14, itmax=400)
    assert rel(s, gold["sigma_plain"]) < 1e-12
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, 1e-9, 8)
    s, st = bie.gpu_solve(op, f, rtol=1e-14, itmax=400)
    assert rel(s, gold["sigma_corrected"]) < 1e-12
    src = [bie.PointSource(tuple(p), float(c)) for p, c in zip(gold["block_src"], gold["block_q"])]
    F = bie.rhs_dielectric_box3d(itf, src, 4.0)
    S, st = bie.gpu_solve(op, F, rtol=1e-14, itmax=400)
    for c in range(F.shape[1]):
        assert rel(S[:, c], gold["sigma_block"][:, c]) < 1e-12
    S, st = bie.gpu_solve(op, F, rtol=1e-11, itmax=400, precision="fp32")
    for c in range(F.shape[1]):
        assert rel(S[:, c], gold["sigma_block"][:, c]) < 1e-8
