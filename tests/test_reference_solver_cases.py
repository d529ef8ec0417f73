"""Solver cases of the reference's suite (test/solver/dielectric_box3d.jl) restated on the
GPU path: 3 x 3 x 1 box, n_quad = 6, l_ec = 0.2, eps_in = 4, point source at (0.1, 0.1, 0.1),
GMRES to atol = rtol = 1e-6. Each solve leaves a residual below 1e-5 and a total
polarisation charge sum w sigma within 0.1 of 1 - 1/eps_in, uncorrected and corrected
(55-73), and with the edge corrections off and on (236-264)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS_BOX = 4.0


@pytest.fixture(scope="module")
def box(bie):
    itf = bie.single_dielectric_box3d(3.0, 3.0, 1.0, 6, 0.2, EPS_BOX, 1.0)
    rhs = bie.rhs_dielectric_box3d(itf, bie.PointSource((0.1, 0.1, 0.1), 1.0), EPS_BOX)
    return itf, rhs


def check(itf, op, rhs, bie):
    x = bie.solve_gmres(op, rhs, 1e-6, 1e-6)
    assert np.linalg.norm(op @ x - rhs) < 1e-5
    err = abs(np.dot(itf.weights, x) + 1.0 / EPS_BOX - 1.0)
    assert err < 1e-1
    return err


def test_dielectric_box3d_corrected_and_uncorrected(bie, box):
    itf, rhs = box
    check(itf, bie.lhs_dielectric_box3d_fmm3d(itf, 1e-6), rhs, bie)
    check(itf, bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-6, 1e-6, 12), rhs, bie)


def test_dielectric_box3d_corrected_edges_flag(bie, box):
    itf, rhs = box
    check(itf, bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-6, 1e-6, 12, correct_edges=False), rhs, bie)
    check(itf, bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-6, 1e-6, 12, correct_edges=True,
                                                        adaptive_atol=1e-6), rhs, bie)
