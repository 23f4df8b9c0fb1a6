"""Rasters of any width against the oracle: the transform along x for widths whose half is not a
power of two (mixed-radix passes when every prime factor of w is at most 64, Bluestein's chirp
z-transform otherwise), with the height on the cosine transform or the row solve.

The reference plans its FFT at any length (Spectral::new, flexure.rs:1139-1170), and coarsening
(flexure.rs:2110-2121) only asks the solve's width to be a multiple of 2f with w/f >= 16, so
widths such as 48, 96, 1536 or 3000 reach Solver::solve. Tolerances as the other flexure tests:
the mean-D preconditioner's transforms are FP64 kernels, compared at 1e-10 relative (the bank's
sqrt weights amplify ulp differences, 1e-8); FP32 transforms at 5e-5; solves to relative
residual 1e-10 against the oracle's to 1e-12 at relative L2 1e-8.
"""
import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import _lib as L
from deeptime_gpu import flexure as F
from deeptime_gpu import inputs as I

pytestmark = pytest.mark.gpu
RHO_M = 3300.0


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# (w, h): smooth widths (2, 3, 5 and 7 factors), odd ones, a prime factor above 64 (Bluestein:
# 67, 257 and 2 x 131), and a height off the power-of-two transform (the row solve)
WIDTHS = [(48, 16), (96, 40), (75, 32), (6, 8), (7, 5), (67, 16), (257, 64), (262, 32), (1536, 512), (3000, 1000)]


@pytest.mark.parametrize("w,h", WIDTHS)
def test_the_preconditioner_matches_the_oracle_at_any_width(w, h):
    dx = 20_000.0
    d, c, _ = I.flexure_problem(w, h, 4.0, w + 7 * h)
    r = np.random.default_rng(w * h).standard_normal((h, w)) * 1e4
    sv = F.Solver(w, h, dx)
    for precond in (L.PRECOND_MEAN_D, L.PRECOND_REFERENCE):
        want = O.flex_precondition(d, c, r, dx, precond)
        z = sv.precondition(d, c, r, precond, L.PREC_FP64)
        assert rel_l2(z, want) < (1e-10 if precond == L.PRECOND_MEAN_D else 1e-8), (w, h, precond)
        z32 = sv.precondition(d, c, r, precond, L.PREC_MIXED)
        assert rel_l2(z32, want) < 5e-5, (w, h, precond)


@pytest.mark.parametrize("w,h", [(48, 16), (96, 40), (75, 32), (67, 16), (257, 64), (1536, 512), (3000, 1000)])
def test_solves_at_any_width_match_the_oracle(w, h):
    dx = 10_000.0
    d, c, b = I.flexure_problem(w, h, 4.0, 11 * w + h)
    xo, ro = O.flex_solve(d, c, b, dx, 1e-12, 20000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
    assert ro["converged"]
    sv = F.Solver(w, h, dx)
    for prec in (L.PREC_FP64, L.PREC_MIXED_RELIABLE):
        x, rep = sv.solve_with(d, c, b, F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=prec,
                                                 tol=1e-10, max_iterations=20000))
        assert rep.converged and rep.rel_residual <= 1e-10, (w, h, prec, rep)
        assert rel_l2(x, xo) < 1e-8, (w, h, prec)


def test_the_reference_rule_at_a_coarsened_width_matches_the_oracle():
    # a raster of 3000 x 1500 cells of 15 km coarsened by 2 (coarsening keeps the solve cell at or
    # under 45 km): the solve runs at 1500 x 750, 30 km, with the reference's max|z| < 2 m rule
    w, h, dx = 1500, 750, 30_000.0
    d, c, _ = I.flexure_problem(w, h, 4.0, 1500)
    b = np.zeros((h, w))
    b.ravel()[::89] = RHO_M * 2500.0
    x, rep = F.Solver(w, h, dx).solve(d, c, b, 2.0, 60)
    xo, ro = O.flex_solve(d, c, b, dx, 2.0, 60)
    assert rep.converged and ro["converged"], (rep, ro)
    assert abs(rep.iterations - ro["iterations"]) <= 1, (rep, ro)
    assert rel_l2(x, xo) < 1e-6
