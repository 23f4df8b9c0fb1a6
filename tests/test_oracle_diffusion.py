"""Pins the CPU oracle's diffusion solves to the reference's own tests
(crates/deeptime-core/src/surface/diffusion/multigrid/tests.rs and surface/diffusion.rs tests)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.fixtures import SIZES, diffusion_bound, rms, shelf_kd, submarine_kd, terrain


def test_submarine_kd_matches_the_oracle():
    for z in (-5.0, 0.0, 1.0, 30.0, 61.0, 500.0):
        a = O.submarine_kd(z, 100.0, 60.0, 2.0, 3.0)
        b = float(submarine_kd(np.array(z), 100.0, 60.0, 2.0, 3.0))
        assert a == pytest.approx(b, rel=1e-15, abs=1e-15)


def test_cyclic_solves_a_ring():
    # surface/diffusion.rs:1083-1105
    n = 5
    k = [0.3, 1.2, 0.7, 2.0, 0.1]
    lo = np.array([-k[(i + n - 1) % n] for i in range(n)])
    up = np.array([-k[i] for i in range(n)])
    di = 1.0 - lo - up
    b0 = np.array([1.0, -2.0, 3.0, 0.5, 4.0])
    x = O.cyclic(lo, di, up, up[n - 1], lo[0], b0)
    for i in range(n):
        ax = di[i] * x[i] + lo[i] * x[(i + n - 1) % n] + up[i] * x[(i + 1) % n]
        assert abs(ax - b0[i]) < 1e-10


def test_the_operator_is_the_definitions():
    for w, h in [(1, 1), (2, 5), (17, 9), (64, 40)]:
        for wrap in (True, False):
            b = terrain(w, h, 3 + w)
            kd = shelf_kd(b, 2)
            x = np.random.default_rng(w).standard_normal((h, w))
            y1 = O.diff_operator(x, kd, 2.0e6, 2400.0, wrap)
            y2 = O.diff_apply_reference(x, kd, 2.0e6, 2400.0, wrap)
            assert np.max(np.abs(y1 - y2)) <= 1e-12 * max(1.0, np.max(np.abs(y2)))


def test_the_multigrid_solve_meets_its_tolerance_and_keeps_the_mass():
    # multigrid/tests.rs:182-217
    solved = 0
    for w, h in SIZES:
        for wrap in (True, False):
            for seed in (1, 2):
                b = terrain(w, h, seed * 7 + w)
                kd = shelf_kd(b, seed)
                for dt, tol in [(2.0e6, 1.0e-6), (2.0e6, 1.0e-3), (2.0e4, 1.0e-6)]:
                    exact = O.diff_reference_cg(b, kd, dt, 2400.0, wrap)
                    x, its, _ = O.diff_solve_mg(b, kd, dt, 2400.0, tol, wrap)
                    assert its < 400
                    e, s, g = O.diff_operator_coeffs(kd, dt, 2400.0, wrap)
                    lim = diffusion_bound(e, s, g, tol)
                    assert rms(x, exact) <= lim, (w, h, wrap, seed, dt, tol)
                    sb, sx = b.sum(), x.sum()
                    assert abs(sb - sx) <= 1e-12 * max(np.abs(b).sum(), 1.0)
                    x0, _, _ = O.diff_solve_mg(b, kd, dt, 2400.0, tol, wrap, use_lod=False)
                    assert rms(x0, exact) <= lim
                    solved += 1
    assert solved >= 100


def test_the_multigrid_and_jacobi_solves_agree_within_their_tolerance():
    # multigrid/tests.rs:220-238
    for w, h in [(64, 40), (129, 67), (5, 3)]:
        for wrap in (True, False):
            b = terrain(w, h, 11 + w)
            kd = shelf_kd(b, 3)
            dt, tol = 2.0e6, 1.0e-6
            xm, _, _ = O.diff_solve_mg(b, kd, dt, 2400.0, tol, wrap)
            xj, _ = O.diff_solve_jacobi(b, kd, dt, 2400.0, wrap)
            e, s, g = O.diff_operator_coeffs(kd, dt, 2400.0, wrap)
            assert rms(xm, xj) <= 2.0 * diffusion_bound(e, s, g, tol)


@pytest.mark.parametrize("cycle", [O.CYCLE_JACOBI, O.CYCLE_RBGS])
def test_the_cycle_is_a_symmetric_positive_definite_operator(cycle):
    # multigrid/tests.rs:243-289 (and the same property for the benchmark's red-black cycle)
    for w, h, wrap in [(64, 40, True), (37, 23, False), (5, 3, True), (2, 9, True), (1, 1, False), (64, 32, True)]:
        z = terrain(w, h, 5)
        kd = shelf_kd(z, 5)
        rng = np.random.default_rng(9)
        r1 = rng.random((h, w)) - 0.5
        r2 = rng.random((h, w)) - 0.5
        z1, rz1, _ = O.diff_vcycle(r1, kd, 2.0e6, 2400.0, wrap, cycle)
        z2, rz2, _ = O.diff_vcycle(r2, kd, 2.0e6, 2400.0, wrap, cycle)
        z1, z2 = z1.astype(np.float64), z2.astype(np.float64)
        assert rz1 > 0 and rz2 > 0
        assert abs(rz1 - (z1 * r1).sum()) <= 1e-9 * abs(rz1)
        a, b = (z1 * r2).sum(), (r1 * z2).sum()
        assert abs(a - b) <= 1e-4 * np.sqrt(rz1 * rz2), (w, h, a, b)


def test_the_cycle_takes_far_fewer_iterations_than_jacobi_on_a_shelf():
    # multigrid/tests.rs:292-301
    w, h = 256, 128
    b = terrain(w, h, 21)
    kd = shelf_kd(b, 21)
    _, mg, _ = O.diff_solve_mg(b, kd, 2.0e6, 2400.0, 1.0e-6, True)
    _, jac = O.diff_solve_jacobi(b, kd, 2.0e6, 2400.0, True)
    assert 3 * mg <= jac, (mg, jac)


@pytest.mark.parametrize("precision", [32, 64])
def test_the_red_black_cycle_solves_to_a_relative_residual(precision):
    # the benchmark's variant: V(2,2) red-black Gauss-Seidel to 16 x 8, relative residual 1e-10.
    w, h = 128, 64
    b = terrain(w, h, 4)
    kd = shelf_kd(b, 4)
    x, its, rel = O.diff_solve_mg(b, kd, 2.0e6, 2400.0, 1e-10, True, stop=O.STOP_REL_RESIDUAL, cycle=O.CYCLE_RBGS,
                                  precision=precision)
    assert its < 60 and rel < 1e-9, (its, rel)
    _, nl = O.diff_vcycle(b, kd, 2.0e6, 2400.0, True, O.CYCLE_RBGS)[1:], None
    exact = O.diff_reference_cg(b, kd, 2.0e6, 2400.0, True)
    assert np.linalg.norm(x - exact) / np.linalg.norm(exact) < 1e-9
