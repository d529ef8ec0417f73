"""End-to-end accuracy near a box corner, the reference's test
"correct_edges improves edge-near pointwise potential" (test/solver/dielectric_box3d.jl:279-322):
a 3 x 3 x 1 box (n_quad = 6, eps_in = 4) with a point source inside, solved by GMRES on the
GPU to 1e-7 with the edge corrections off and on at l_ec = 0.10, against a solve with
corrections at l_ec = 0.06. The potential at (1.40, 1.40, 0.40) is the source's plus the
induced single layer evaluated like laplace3d_pottrg_near (adaptive near panels). The
reference's bars: the corrected error below half the uncorrected one and below 1e-4."""
import math

import numpy as np
import pytest

from probe_reference import pottrg_near

pytestmark = pytest.mark.gpu

EPS_BOX = 4.0
SOURCE = (0.1, 0.1, 0.1)
TARGET = np.array([1.40, 1.40, 0.40])


def potential(bie, l_ec, correct_edges):
    itf = bie.single_dielectric_box3d(3.0, 3.0, 1.0, 6, l_ec, EPS_BOX, 1.0)
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-6, 1e-6, 12, correct_edges=correct_edges,
                                                  adaptive_atol=1e-8)
    rhs = bie.rhs_dielectric_box3d(itf, bie.PointSource(SOURCE, 1.0), EPS_BOX)
    sigma = bie.solve_gmres(op, rhs, 1e-7, 1e-7)
    r = math.dist(TARGET, SOURCE)
    return 1.0 / (4 * math.pi * r) / EPS_BOX + pottrg_near(itf, sigma, TARGET, 5.0)


def test_edge_corrections_improve_the_near_corner_potential(bie):
    ref = potential(bie, 0.06, True)
    err_off = abs(potential(bie, 0.10, False) - ref)
    err_on = abs(potential(bie, 0.10, True) - ref)
    assert err_on < err_off / 2, (err_on, err_off)
    assert err_on < 1e-4, (err_on, err_off)
