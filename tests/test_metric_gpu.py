"""The sphere's row metric on the device (RowMetric / RowSolve, flexure.rs:954-1099), through the
C ABI, against the CPU oracle's restatement of the same.

Tolerances as the block metric's tests: the operator is an FP64 stencil, compared at 1e-12
relative; the preconditioner (the row solve per wavenumber in place of the cosine transform) at
1e-10 relative for the mean level and 1e-8 for the bank's blend (whose weights are sensitive at
the nodes), 5e-5 in FP32; converged solves by their relative L2 distance, at most 1e-8, when both are
solved to a relative residual well below it.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import _lib as L
from deeptime_gpu import flexure as F

pytestmark = pytest.mark.gpu
G = 9.81
RHO_M = 3300.0
RHO_W = O.RHO_WATER


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def sphere_faces(h, dx, r_m):
    # the sines of latitude at the rows' boundaries of an equal-area raster (flexure.rs:5341-5345)
    k = np.arange(h + 1)
    return np.clip((0.5 * h - k) * dx / r_m, -1.0, 1.0)


def metric_for(h, dx, span=0.49):
    return O.row_metric_from_sin_faces(sphere_faces(h, dx, span * h * dx), 1)


def plate(w, h, seed):
    rng = np.random.default_rng(seed)
    j, i = np.mgrid[0:h, 0:w]
    te = np.where(((i // 12) + (j // 9)) % 3 == 0, 60.0, 8.0)
    te = O.box_blur(te, 2, 2, wrap=True)
    d = np.vectorize(lambda t: O.rigidity_per_g(t, G))(te)
    c = np.where(i < w // 3, RHO_M - RHO_W, RHO_M).astype(np.float64)
    b = rng.standard_normal((h, w)) * 1e4
    return d, c, b


@pytest.mark.parametrize("w,h", [(64, 32), (128, 64), (256, 32)])
def test_operator_and_bend_on_the_sphere_match_the_oracle(w, h):
    dx = 50_000.0
    metric = metric_for(h, dx)
    d, c, _ = plate(w, h, w + h)
    v = np.random.default_rng(h).standard_normal((h, w)) * 100.0
    sv = F.Solver(w, h, dx, metric)
    assert rel_l2(sv.operator(d, c, v), O.flex_operator(d, c, v, dx, metric)) < 1e-12
    # bend = L (d L v): the operator with c = 0
    assert rel_l2(sv.bend(d, v), O.flex_operator(d, np.zeros_like(c), v, dx, metric)) < 1e-12


@pytest.mark.parametrize("precond", [L.PRECOND_REFERENCE, L.PRECOND_MEAN_D])
@pytest.mark.parametrize("w,h", [(128, 64), (64, 41), (128, 300)])
def test_the_row_solve_preconditioner_matches_the_oracle(precond, w, h):
    # h = 41: on the row metric the raster's height need not be a power of two; h = 300: the
    # row solve runs in chunks of 64 rows (the last one of 44)
    dx = 50_000.0
    metric = metric_for(h, dx)
    d, c, r = plate(w, h, 7)
    sv = F.Solver(w, h, dx, metric)
    z = sv.precondition(d, c, r, precond=precond)
    want = O.flex_precondition(d, c, r, dx, precond, metric)
    # The bank's blend weights move by up to 1e-9 where a cell sits within an ulp of a node (the
    # block metric's test says why), so the blend is compared at 1e-8; the mean level at 1e-10.
    bound = 1e-10 if precond == L.PRECOND_MEAN_D else 1e-8
    assert rel_l2(z, want) < bound
    z32 = sv.precondition(d, c, r, precond=precond, precision=L.PREC_MIXED)
    assert rel_l2(z32, want) < 5e-5


def test_uniform_plate_on_the_sphere_is_solved_by_its_preconditioner():
    # flexure.rs:5388-5432: with uniform d and c the row solve is the exact inverse, one iteration
    w, h, dx = 64, 32, 50_000.0
    metric = metric_for(h, dx)
    _, _, b = plate(w, h, 3)
    d = np.full((h, w), O.rigidity_per_g(25.0, G))
    c = np.full((h, w), RHO_M)
    sv = F.Solver(w, h, dx, metric)
    x, rep = sv.solve(d, c, b, 1e-9, 20)
    assert rep.iterations <= 1, rep
    ax = O.flex_operator(d, c, x, dx, metric)
    assert np.abs(ax - b).max() < 1e-9 * np.abs(b).max()


def test_block_couplings_through_the_row_solve_give_the_cosine_transform_answer():
    # flexure.rs:5433-5444: RowMetric::block(h) on the row-solve path equals the block metric
    w, h, dx = 128, 64, 20_000.0
    block = (np.ones(h), np.array([0.0] + [1.0] * (h - 1) + [0.0]))
    d, c, b = plate(w, h, 5)
    p = F.params(stop=L.STOP_REL_RESIDUAL, tol=1e-11, max_iterations=400)
    xr, rr = F.Solver(w, h, dx, block).solve_with(d, c, b, p)
    xb, rb = F.Solver(w, h, dx).solve_with(d, c, b, p)
    assert rr.converged and rb.converged
    assert rel_l2(xr, xb) < 1e-9


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED, L.PREC_MIXED_RELIABLE])
@pytest.mark.parametrize("w,h", [(256, 128), (128, 82)])
def test_solve_on_the_sphere_matches_the_oracle(precision, w, h):
    dx = 40_000.0
    metric = metric_for(h, dx)
    d, c, b = plate(w, h, 11)
    want, orep = O.flex_solve(d, c, b, dx, 1e-12, 2000, stop=L.STOP_REL_RESIDUAL, metric=metric)
    assert orep["converged"], orep
    sv = F.Solver(w, h, dx, metric)
    p = F.params(stop=L.STOP_REL_RESIDUAL, precision=precision, tol=1e-10, max_iterations=2000)
    x, rep = sv.solve_with(d, c, b, p)
    assert rep.converged, rep
    # the stop rule reads the recurrence's residual; the report's is recomputed from x
    assert rep.rel_residual < 2e-10, rep
    assert rel_l2(x, want) < 1e-8


def test_a_metric_needs_both_couplings():
    a = np.ones(8)
    h = ctypes.c_void_p()
    st = L.lib().dt_flex_create(16, 8, 1000.0, ctypes.c_void_p(a.ctypes.data), None, ctypes.byref(h))
    assert st == L.DT_BAD_ARG and not h.value
    # any width and any height
    for w in (24, 16):
        st = L.lib().dt_flex_create(w, 41, 1000.0, None, None, ctypes.byref(h))
        assert st == L.DT_OK and h.value
        L.lib().dt_flex_destroy(h)
