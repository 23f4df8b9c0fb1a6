"""Parity of the device flexure solve with the CPU oracle, through the C ABI (libdeeptime_gpu.so).

Tolerances: the operator and transforms are FP64 kernels, compared at 1e-12 relative (different
operation order and fused multiply-adds, nothing else); converged solves are compared by their
relative L2 distance, at most 1e-8 (the benchmark's bar) when both are solved well below it.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import _lib as L
from deeptime_gpu import flexure as F
from deeptime_gpu import inputs as I

pytestmark = pytest.mark.gpu
G = 9.81
RHO_M = 3300.0


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def patchy(w, h, lo, hi):
    j, i = np.mgrid[0:h, 0:w]
    te = np.where(((i // 24) + (j // 24)) % 3 == 0, hi, lo).astype(np.float64)
    return O.box_blur(te, 2, 2, wrap=True)


def rigidity(te):
    return np.vectorize(lambda t: O.rigidity_per_g(t, G))(te)


@pytest.fixture(scope="module")
def problem():
    w, h, dx = 128, 64, 20_000.0
    d = rigidity(patchy(w, h, 5.0, 60.0))
    c = np.where(np.arange(w)[None, :] < w // 3, RHO_M - 1030.0, RHO_M) * np.ones((h, 1))
    rng = np.random.default_rng(1)
    return w, h, dx, d, c, rng


def test_the_device_reports_itself():
    assert L.device_info() is not None


@pytest.mark.parametrize("w,h", [(16, 8), (128, 64), (256, 128), (16, 1024), (512, 32)])
def test_operator_and_bend_match_the_oracle(w, h):
    dx = 10_000.0
    rng = np.random.default_rng(w + h)
    d = 10.0 ** (21 + 3 * rng.random((h, w))) / G
    c = np.full((h, w), RHO_M)
    v = rng.standard_normal((h, w)) * 100.0
    sv = F.Solver(w, h, dx)
    y = sv.operator(d, c, v)
    want = O.flex_operator(d, c, v, dx)
    assert rel_l2(y, want) < 1e-13
    yb = sv.bend(d, v)
    wb = O.flex_bend(d, v, dx)
    assert rel_l2(yb, wb) < 1e-13


@pytest.mark.parametrize("precond", [L.PRECOND_MEAN_D, L.PRECOND_REFERENCE])
def test_preconditioner_matches_the_oracle(problem, precond):
    w, h, dx, d, c, rng = problem
    r = rng.standard_normal((h, w)) * 1e4
    sv = F.Solver(w, h, dx)
    z = sv.precondition(d, c, r, precond, L.PREC_FP64)
    want = O.flex_precondition(d, c, r, dx, precond)
    # The bank's blend weights are sqrt(f) of the cell's place between two nodes
    # (flexure.rs:1393-1396). The box-blurred plate leaves thousands of cells within 1e-12 of a
    # node, where one ulp of ln(alpha) (the device's log/pow against the host's) moves the weight
    # by up to 1e-9; the blend then differs at 1e-10 relative. The mean level has no weights.
    bound = 1e-12 if precond == L.PRECOND_MEAN_D else 1e-8
    assert rel_l2(z, want) < bound
    z32 = sv.precondition(d, c, r, precond, L.PREC_MIXED)
    assert rel_l2(z32, want) < 5e-5


@pytest.mark.parametrize("w,h", [(4, 2), (8, 4), (32, 2), (2, 16)])
def test_transforms_on_tiny_rasters(w, h):
    dx = 10_000.0
    rng = np.random.default_rng(3)
    d = np.full((h, w), 1e21)
    c = np.full((h, w), RHO_M)
    r = rng.standard_normal((h, w))
    z = F.Solver(w, h, dx).precondition(d, c, r, L.PRECOND_MEAN_D)
    assert rel_l2(z, O.flex_precondition(d, c, r, dx, O.PRECOND_MEAN_D)) < 1e-12


def test_a_point_load_sinks_by_the_analytic_depth_on_the_device():
    # flexure.rs:2810-2853 through the device solve (reference preconditioner and rule)
    w, h, dx = 256, 128, 10_000.0
    d = np.full((h, w), O.rigidity_per_g(30.0, G))
    c = np.full((h, w), RHO_M)
    l = (d[0, 0] / RHO_M) ** 0.25
    mass = 1.0e15
    b = np.zeros((h, w))
    b[h // 2, w // 2] = mass / (dx * dx)
    x, rep = F.Solver(w, h, dx).solve(d, c, b, 1e-9, 50)
    assert rep.converged and rep.iterations <= 1, rep
    analytic = mass / (8.0 * RHO_M * l * l)
    assert abs(x[h // 2, w // 2] / analytic - 1.0) < 0.03
    assert abs(x.sum() * RHO_M * dx * dx / mass - 1.0) < 1e-9
    assert -0.05 * analytic < x.min() < 0.0
    xo, _ = O.flex_solve(d, c, b, dx, 1e-9, 50)
    assert rel_l2(x, xo) < 1e-10


def test_a_line_load_gives_the_analytic_profile_on_the_device():
    # flexure.rs:2890-2931 (its first checks) on 16 x 1024
    w, h, dx = 16, 1024, 5000.0
    d = np.full((h, w), O.rigidity_per_g(30.0, G))
    c = np.full((h, w), RHO_M)
    alpha = O.flexural_parameter_m(d[0, 0])
    b = np.zeros((h, w))
    b[h // 2, :] = 1.0e10 / dx
    x, rep = F.Solver(w, h, dx).solve(d, c, b, 1e-9, 50)
    assert rep.converged
    profile = x[h // 2:, 0]
    assert abs(profile[0] / (1.0e10 / (2.0 * RHO_M * alpha)) - 1.0) < 0.01
    k = int(np.argmax(profile < 0.0))
    zero = (k - 1.0 + profile[k - 1] / (profile[k - 1] - profile[k])) * dx
    assert abs(zero / (0.75 * math.pi * alpha) - 1.0) < 0.02


def test_the_reference_rule_matches_the_oracle_on_a_patchy_plate(problem):
    # the production call: tolerance 2 m, at most 60 iterations, reference preconditioner
    w, h, dx, d, c, rng = problem
    b = np.zeros((h, w))
    b.ravel()[::37] = RHO_M * 2000.0
    x, rep = F.Solver(w, h, dx).solve(d, c, b, 0.01, 400)
    xo, ro = O.flex_solve(d, c, b, dx, 0.01, 400)
    assert rep.converged and ro["converged"]
    assert abs(rep.iterations - ro["iterations"]) <= 1, (rep, ro)
    assert rel_l2(x, xo) < 1e-6
    assert abs((x * c).sum() / b.sum() - 1.0) < 1e-3


def test_the_solve_is_stable_at_the_editors_extremes_on_the_device():
    # flexure.rs:3146-3164
    w, h, dx = 128, 64, 39_000.0
    sv = F.Solver(w, h, dx)
    for lo, hi in [(1.25, 20.0), (15.0, 240.0), (0.1, 1.0), (300.0, 500.0)]:
        d = rigidity(patchy(w, h, lo, hi))
        c = np.full((h, w), RHO_M)
        b = np.zeros(w * h)
        b[::53] = RHO_M * 3000.0
        b = b.reshape(h, w)
        x, rep = sv.solve(d, c, b, 0.1, 400)
        assert rep.converged, (lo, hi, rep)
        assert np.all(np.isfinite(x))
        assert abs(x.sum() * RHO_M / b.sum() - 1.0) < 1e-3


@pytest.mark.parametrize("precond", [L.PRECOND_MEAN_D, L.PRECOND_REFERENCE])
def test_baseline_plain_fp64_matches_the_oracle(precond):
    # the 512 x 256 workload at 10 km, sigma 8 cells: PCG to 1e-10 against the oracle at 1e-12
    w, h, dx = 512, 256, 10_000.0
    d, c, b = I.flexure_problem(w, h, 8.0, 1000)
    xo, ro = O.flex_solve(d, c, b, dx, 1e-12, 5000, precond=O.PRECOND_MEAN_D, stop=O.STOP_REL_RESIDUAL)
    assert ro["converged"]
    sv = F.Solver(w, h, dx)
    p = F.params(precond=precond, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_FP64, tol=1e-10, max_iterations=5000)
    x, rep = sv.solve_with(d, c, b, p)
    assert rep.converged, rep
    assert rep.rel_residual < 2e-10
    assert rel_l2(x, xo) < 1e-8


@pytest.mark.parametrize("precision", [L.PREC_MIXED, L.PREC_MIXED_RELIABLE])
@pytest.mark.parametrize("precond", [L.PRECOND_MEAN_D, L.PRECOND_REFERENCE])
def test_mixed_precision_reaches_the_fp64_answer(precond, precision):
    # FP32 PCG inside FP64 refinement, or with FP64 reliable updates, to 1e-8 at the fine-grid
    # conditioning (dx 2.5 km)
    w, h, dx = 512, 256, 2500.0
    d, c, b = I.flexure_problem(w, h, 32.0, 1200)
    xo, ro = O.flex_solve(d, c, b, dx, 1e-12, 10000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
    sv = F.Solver(w, h, dx)
    p = F.params(precond=precond, stop=L.STOP_REL_RESIDUAL, precision=precision, tol=1e-8, max_iterations=20000)
    x, rep = sv.solve_with(d, c, b, p)
    assert rep.converged, rep
    assert rep.rel_residual <= 1e-8
    assert rel_l2(x, xo) < 1e-8


def test_reliable_updates_take_about_the_fp64_iterations():
    # one FP32 Krylov sequence with FP64 residual replacements: no restarts, so the iteration count
    # stays near the FP64 solve's (refinement restarts and needs more)
    w, h, dx = 512, 256, 2500.0
    d, c, b = I.flexure_problem(w, h, 32.0, 1201)
    sv = F.Solver(w, h, dx)
    its = {}
    for precision in (L.PREC_FP64, L.PREC_MIXED_RELIABLE):
        p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=precision, tol=1e-8,
                     max_iterations=20000)
        x, rep = sv.solve_with(d, c, b, p)
        assert rep.converged and rep.rel_residual <= 1e-8
        its[precision] = rep.iterations
    print(its)
    assert its[L.PREC_MIXED_RELIABLE] <= 1.25 * its[L.PREC_FP64] + 2, its


def test_a_given_first_guess_is_kept_only_when_it_beats_zero():
    w, h, dx = 128, 64, 10_000.0
    d, c, b = I.flexure_problem(w, h, 8.0, 7)
    sv = F.Solver(w, h, dx)
    p = F.params(precond=L.PRECOND_MEAN_D, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=3000,
                 warm_start=L.WARM_GIVEN)
    x_exact, _ = sv.solve_with(d, c, b, F.params(precond=L.PRECOND_MEAN_D, stop=L.STOP_REL_RESIDUAL, tol=1e-12,
                                                   max_iterations=3000))
    good = x_exact * (1.0 + 1e-3)
    x, rep = sv.solve_with(d, c, b, p, x0=good)
    assert rep.warm_start_accepted and rep.warm_start_rel_residual < 1e-2 and rep.converged
    bad = x_exact * -3.0
    x2, rep2 = sv.solve_with(d, c, b, p, x0=bad)
    assert not rep2.warm_start_accepted and rep2.converged
    assert rel_l2(x2, x_exact) < 1e-8


def test_non_finite_input_is_reported():
    w, h, dx = 64, 32, 10_000.0
    d = np.full((h, w), 1e22)
    c = np.full((h, w), RHO_M)
    b = np.ones((h, w))
    b[3, 4] = np.nan
    sv = F.Solver(w, h, dx)
    with pytest.raises(L.DeepTimeError) as e:
        sv.solve_with(d, c, b, F.params(stop=L.STOP_REL_RESIDUAL, tol=1e-8, max_iterations=50))
    assert e.value.status == L.DT_NONFINITE


def test_the_iteration_cap_reports_not_converged():
    w, h, dx = 128, 64, 10_000.0
    d, c, b = I.flexure_problem(w, h, 8.0, 9)
    x, rep = F.Solver(w, h, dx).solve_with(d, c, b, F.params(precond=L.PRECOND_MEAN_D, stop=L.STOP_REL_RESIDUAL,
                                                              tol=1e-14, max_iterations=3))
    assert not rep.converged and rep.iterations == 3 and rep.status == L.DT_NOT_CONVERGED


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("w,h", [(16384, 64), (128, 8192)])
def test_the_longest_transforms_match_the_oracle(w, h, precision):
    # rows of 8192 complex values (w = 16384) and columns of 8192: the lengths of the 16384 x 8192
    # timestep raster, on thin rasters the oracle solves in seconds
    dx = 1250.0
    d, c, _ = I.flexure_problem(w, h, 8.0, 77)
    r = np.random.default_rng(w).standard_normal((h, w)) * 1e4
    sv = F.Solver(w, h, dx)
    for precond in (L.PRECOND_MEAN_D, L.PRECOND_REFERENCE):
        z = sv.precondition(d, c, r, precond, precision)
        want = O.flex_precondition(d, c, r, dx, precond)
        bound = (1e-12 if precond == L.PRECOND_MEAN_D else 1e-8) if precision == L.PREC_FP64 else 5e-5
        assert rel_l2(z, want) < bound, (precond, rel_l2(z, want))


@pytest.mark.parametrize("w,h", [(64, 41), (128, 82), (256, 300)])
def test_heights_that_are_not_powers_of_two_match_the_oracle(w, h):
    # The block metric at a height the cosine transform does not take: along y each wavenumber
    # is solved by the row solve with the block metric's couplings (RowMetric::block,
    # flexure.rs:1000-1010), which is that transform's inverse; the Jacobi weights stay the block
    # metric's. The oracle takes its own Bluestein route for such heights.
    dx = 20_000.0
    d = rigidity(patchy(w, h, 5.0, 60.0))
    c = np.where(np.arange(w)[None, :] < w // 3, RHO_M - 1030.0, RHO_M) * np.ones((h, 1))
    r = np.random.default_rng(h).standard_normal((h, w)) * 1e4
    sv = F.Solver(w, h, dx)
    for precond in (L.PRECOND_MEAN_D, L.PRECOND_REFERENCE):
        want = O.flex_precondition(d, c, r, dx, precond)
        z = sv.precondition(d, c, r, precond, L.PREC_FP64)
        assert rel_l2(z, want) < (1e-10 if precond == L.PRECOND_MEAN_D else 1e-8), precond
        z32 = sv.precondition(d, c, r, precond, L.PREC_MIXED)
        assert rel_l2(z32, want) < 5e-5, precond


def test_the_production_raster_takes_the_reference_rule_like_the_oracle():
    # the timestep's flexure raster (1024 x 328 at the reference's 39 km cells): the max|z| rule
    # at 2 m, 60 iterations, the reference preconditioner
    w, h, dx = 1024, 328, 39_000.0
    d, c, _ = I.flexure_problem(w, h, 8.0, 328)
    b = np.zeros((h, w))
    b.ravel()[::97] = RHO_M * 2500.0
    x, rep = F.Solver(w, h, dx).solve(d, c, b, 2.0, 60)
    xo, ro = O.flex_solve(d, c, b, dx, 2.0, 60)
    assert rep.converged and ro["converged"], (rep, ro)
    assert abs(rep.iterations - ro["iterations"]) <= 1, (rep, ro)
    assert rel_l2(x, xo) < 1e-6
