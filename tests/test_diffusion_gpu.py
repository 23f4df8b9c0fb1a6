"""Parity of the device diffusion solve with the CPU oracle, through the C ABI.

Ports of crates/deeptime-core/src/surface/diffusion/multigrid/tests.rs run on the device (same
sizes, seeds, tolerances and bounds), plus the benchmark's variants against the oracle. The cycle runs
in FP32 (as the reference's), so cycles are compared at 1e-4 of the reference's own symmetric
tolerance scale, and solves by the reference's error bound.
"""
import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import _lib as L
from deeptime_gpu import diffusion as D
from deeptime_gpu import inputs as I
from tests.fixtures import SIZES, diffusion_bound, rms, shelf_kd, terrain

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("w,h,wrap", [(1, 1, False), (2, 5, True), (17, 9, True), (64, 40, False), (256, 128, True)])
def test_operator_matches_the_oracle(w, h, wrap):
    b = terrain(w, h, 3 + w)
    kd = shelf_kd(b, 2)
    x = np.random.default_rng(w).standard_normal((h, w))
    ws = D.Workspace(D.Dims(w, h, 2400.0, wrap))
    y = ws.operator(kd, 2.0e6, x)
    assert np.max(np.abs(y - O.diff_operator(x, kd, 2.0e6, 2400.0, wrap))) <= 1e-12 * max(1.0, np.abs(y).max())


@pytest.mark.parametrize("cycle", [L.CYCLE_JACOBI, L.CYCLE_RBGS])
@pytest.mark.parametrize("w,h,wrap", [(64, 40, True), (37, 23, False), (5, 3, True), (2, 9, True), (1, 1, False), (256, 128, True)])
def test_the_cycle_matches_the_oracle(cycle, w, h, wrap):
    z0 = terrain(w, h, 5)
    kd = shelf_kd(z0, 5)
    r = np.random.default_rng(9).random((h, w)) - 0.5
    ws = D.Workspace(D.Dims(w, h, 2400.0, wrap))
    z, levels = ws.vcycle(kd, 2.0e6, r, cycle)
    zo, rzo, levels_o = O.diff_vcycle(r, kd, 2.0e6, 2400.0, wrap, cycle)
    assert levels == levels_o
    # FP32 cycle on both sides; the device fuses multiply-adds
    assert rel_l2(z.astype(np.float64), zo.astype(np.float64)) < 1e-4


@pytest.mark.parametrize("cycle", [L.CYCLE_JACOBI, L.CYCLE_RBGS])
def test_the_device_cycle_is_symmetric_positive_definite(cycle):
    # multigrid/tests.rs:243-289 on the device cycle
    for w, h, wrap in [(64, 40, True), (37, 23, False), (5, 3, True), (2, 9, True)]:
        z0 = terrain(w, h, 5)
        kd = shelf_kd(z0, 5)
        rng = np.random.default_rng(9)
        r1, r2 = rng.random((h, w)) - 0.5, rng.random((h, w)) - 0.5
        ws = D.Workspace(D.Dims(w, h, 2400.0, wrap))
        z1 = ws.vcycle(kd, 2.0e6, r1, cycle)[0].astype(np.float64)
        z2 = ws.vcycle(kd, 2.0e6, r2, cycle)[0].astype(np.float64)
        rz1, rz2 = (z1 * r1).sum(), (z2 * r2).sum()
        assert rz1 > 0 and rz2 > 0
        a, b = (z1 * r2).sum(), (r1 * z2).sum()
        assert abs(a - b) <= 1e-4 * np.sqrt(rz1 * rz2)


def test_the_multigrid_solve_meets_its_tolerance_and_keeps_the_mass():
    # multigrid/tests.rs:182-217 through the device solve
    solved = 0
    for w, h in SIZES:
        for wrap in (True, False):
            ws = D.Workspace(D.Dims(w, h, 2400.0, wrap))
            for seed in (1, 2):
                b = terrain(w, h, seed * 7 + w)
                kd = shelf_kd(b, seed)
                for dt, tol in [(2.0e6, 1.0e-6), (2.0e6, 1.0e-3), (2.0e4, 1.0e-6)]:
                    exact = O.diff_reference_cg(b, kd, dt, 2400.0, wrap)
                    e, s, g = O.diff_operator_coeffs(kd, dt, 2400.0, wrap)
                    lim = diffusion_bound(e, s, g, tol)
                    for guess in (True, False):
                        x, rep = ws.solve_with(b, kd, dt, D.params(tol=tol, first_guess=guess))
                        assert rep.iterations < 400
                        assert rms(x, exact) <= lim, (w, h, wrap, seed, dt, tol, guess)
                        assert abs(b.sum() - x.sum()) <= 1e-12 * max(np.abs(b).sum(), 1.0)
                    solved += 1
    assert solved >= 100


def test_the_reference_entry_point_matches_the_oracle():
    # diffusion::solve(ws, d, h, kd, dt, Multigrid, tol_m): h in place, iterations returned
    d = D.Dims(129, 67, 2400.0, True)
    b = terrain(d.w, d.h, 11)
    kd = shelf_kd(b, 3)
    ws = D.Workspace(d)
    h = b.copy()
    its = D.solve(ws, d, h, kd, 2.0e6, D.MULTIGRID, 1e-6)
    xo, its_o, _ = O.diff_solve_mg(b, kd, 2.0e6, 2400.0, 1e-6, True)
    assert abs(its - its_o) <= 2, (its, its_o)
    e, s, g = O.diff_operator_coeffs(kd, 2.0e6, 2400.0, True)
    assert rms(h, xo) <= 2.0 * diffusion_bound(e, s, g, 1e-6)


def test_the_cycle_takes_far_fewer_iterations_than_jacobi_on_a_shelf():
    # multigrid/tests.rs:292-301: the device solve against the oracle's Jacobi-preconditioned one
    w, h = 256, 128
    b = terrain(w, h, 21)
    kd = shelf_kd(b, 21)
    ws = D.Workspace(D.Dims(w, h, 2400.0, True))
    _, rep = ws.solve_with(b, kd, 2.0e6, D.params(tol=1e-6))
    _, jac = O.diff_solve_jacobi(b, kd, 2.0e6, 2400.0, True)
    assert 3 * rep.iterations <= jac, (rep.iterations, jac)


@pytest.mark.parametrize("precision", [L.DIFF_FP64_CG_FP32_CYCLE, L.DIFF_FP64, L.DIFF_MIXED, L.DIFF_MIXED_RELIABLE])
@pytest.mark.parametrize("cycle", [L.CYCLE_JACOBI, L.CYCLE_RBGS])
def test_baseline_variants_reach_the_fp64_answer(precision, cycle):
    # the 2048 x 1024 workload's recipe at 512 x 256: rel. residual 1e-10 against the oracle's
    # unpreconditioned CG at 1e-13
    w, h = 512, 256
    topo, s = I.diffusion_problem(w, h, 8.0, 4200)
    dx, dt = 1000.0, 1.0
    kd = s * dx * dx / dt  # kappa dt / dx^2 = s
    exact = O.diff_reference_cg(topo, kd, dt, dx, True, rel=1e-13)
    ws = D.Workspace(D.Dims(w, h, dx, True))
    x, rep = ws.solve_with(topo, kd, dt, D.params(cycle=cycle, precision=precision, stop=L.STOP_REL_RESIDUAL, tol=1e-10,
                                                  first_guess=False))
    assert rep.converged and rep.rel_residual < 2e-10, rep
    assert rel_l2(x, exact) < 1e-8
    assert abs(x.sum() - topo.sum()) <= 1e-9 * np.abs(topo).sum()


@pytest.mark.parametrize("stop,tol", [(L.STOP_REL_RESIDUAL, 1e-10), (L.STOP_RMS_RESIDUAL, 1e-6)])
def test_reliable_updates_keep_the_fp64_iteration_count(stop, tol):
    # one FP32 CG whose residual the FP64 b - A x replaces (no restart): no more iterations than
    # FP64 CG plus one, fewer than or as many as FP32 refinement, and the device loop the same
    # iterations and bits as the same kernels driven from the host
    w, h = 512, 256
    topo, s = I.diffusion_problem(w, h, 8.0, 4400)
    kd = s * 1e6
    ws = D.Workspace(D.Dims(w, h, 1000.0, True))
    its = {}
    for name, prec in (("fp64", L.DIFF_FP64), ("refine", L.DIFF_MIXED), ("reliable", L.DIFF_MIXED_RELIABLE)):
        x, rep = ws.solve_with(topo, kd, 1.0, D.params(cycle=L.CYCLE_RBGS, precision=prec, stop=stop, tol=tol))
        assert rep.converged, (name, rep)
        its[name] = rep.iterations
    assert its["reliable"] <= its["fp64"] + 1 and its["reliable"] <= its["refine"], its
    xg, rg = ws.solve_with(topo, kd, 1.0, D.params(cycle=L.CYCLE_RBGS, precision=L.DIFF_MIXED_RELIABLE, stop=stop, tol=tol))
    xh, rh = ws.solve_with(topo, kd, 1.0, D.params(cycle=L.CYCLE_RBGS, precision=L.DIFF_MIXED_RELIABLE, stop=stop, tol=tol,
                                                   host_loop=1))
    assert rg.iterations == rh.iterations and rg.refinements == rh.refinements >= 1, (rg, rh)
    assert np.array_equal(xg, xh)


def test_the_red_black_cycle_needs_fewer_iterations():
    w, h = 512, 256
    topo, s = I.diffusion_problem(w, h, 8.0, 4300)
    kd = s * 1e6
    ws = D.Workspace(D.Dims(w, h, 1000.0, True))
    _, rj = ws.solve_with(topo, kd, 1.0, D.params(cycle=L.CYCLE_JACOBI, stop=L.STOP_REL_RESIDUAL, tol=1e-10))
    _, rg = ws.solve_with(topo, kd, 1.0, D.params(cycle=L.CYCLE_RBGS, stop=L.STOP_REL_RESIDUAL, tol=1e-10))
    assert rg.converged and rj.converged
    assert rg.iterations <= rj.iterations, (rg.iterations, rj.iterations)


@pytest.mark.parametrize("wrap", [True, False])
def test_the_lod_first_guess_matches_the_oracle(wrap):
    # diffusion.rs:370-489: the rows (cyclic when the raster wraps) then the columns, each a
    # tridiagonal solve; the device takes the same operations in the same order
    for w, h in [(64, 32), (257, 129), (2048, 64), (3, 5)]:
        b = terrain(w, h, w + h)
        kd = shelf_kd(b, 2)
        ws = D.Workspace(D.Dims(w, h, 2400.0, wrap))
        got = ws.lod(b, kd, 2.0e6)
        want = O.diff_lod(b, kd, 2.0e6, 2400.0, wrap)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), (w, h, wrap)


@pytest.mark.parametrize("w,h,wrap", [(2048, 1024, True), (257, 129, True), (300, 200, False), (96, 48, True), (64, 40, True),
                                      (41, 9, True)])
def test_the_fused_gauss_seidel_cycle_is_bit_for_bit_the_per_colour_launches(w, h, wrap, monkeypatch):
    # the two sweeps of a level in one tiled launch and the levels of <= 2048 cells in one block
    # (the default) against one launch per colour pass (DT_MG_FUSED=0 at create): the same
    # updates in the same order, so the same bits for the FP32 cycle
    z0 = terrain(w, h, 11)
    kd = shelf_kd(z0, 11)
    r = np.random.default_rng(w + h).random((h, w)) - 0.5
    fused = D.Workspace(D.Dims(w, h, 2400.0, wrap))
    monkeypatch.setenv("DT_MG_FUSED", "0")
    apart = D.Workspace(D.Dims(w, h, 2400.0, wrap))
    monkeypatch.delenv("DT_MG_FUSED")
    for _ in range(2):
        zf, lf = fused.vcycle(kd, 2.0e6, r, L.CYCLE_RBGS)
        za, la = apart.vcycle(kd, 2.0e6, r, L.CYCLE_RBGS)
        assert lf == la and np.array_equal(zf, za), float(np.abs(zf - za).max())
    # solves: the mixed one's FP32 cycle is bit for bit; in FP64 the compiler forms fused
    # multiply-adds differently in the two kernels, so the answers agree to 1e-12 relative
    for precision in (L.DIFF_FP64, L.DIFF_MIXED, L.DIFF_MIXED_RELIABLE):
        p = D.params(cycle=L.CYCLE_RBGS, precision=precision, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=2000)
        xf, rf = fused.solve_with(z0, kd, 2.0e6, p)
        xa, ra = apart.solve_with(z0, kd, 2.0e6, p)
        assert rf.iterations == ra.iterations, (precision, rf.iterations, ra.iterations)
        assert np.abs(xf - xa).max() <= 1e-12 * np.abs(xa).max(), (precision, float(np.abs(xf - xa).max()))


@pytest.mark.parametrize("w,h,wrap", [(2048, 1024, True), (2050, 1030, False), (2000, 1201, False)])
def test_the_large_sweep_tiles_are_bit_for_bit_the_small_ones(w, h, wrap, monkeypatch):
    # k_mg_rb2 on 64 x 32 tiles (FP32 levels of at least four tiles an SM, the default) against
    # 32 x 16 tiles (DT_MG_BIG_TILES=0 at create), on rasters whose last tiles are ragged: the
    # same updates in the same order, so the same bits
    z0 = terrain(w, h, 13)
    kd = shelf_kd(z0, 13)
    r = np.random.default_rng(w * h).random((h, w)) - 0.5
    big = D.Workspace(D.Dims(w, h, 2400.0, wrap))
    monkeypatch.setenv("DT_MG_BIG_TILES", "0")
    small = D.Workspace(D.Dims(w, h, 2400.0, wrap))
    monkeypatch.delenv("DT_MG_BIG_TILES")
    zb, lb = big.vcycle(kd, 2.0e6, r, L.CYCLE_RBGS)
    zs, ls = small.vcycle(kd, 2.0e6, r, L.CYCLE_RBGS)
    assert lb == ls and np.array_equal(zb, zs), float(np.abs(zb - zs).max())
    p = D.params(cycle=L.CYCLE_RBGS, precision=L.DIFF_MIXED_RELIABLE, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=2000)
    xb, rb = big.solve_with(z0, kd, 2.0e6, p)
    xs, rs = small.solve_with(z0, kd, 2.0e6, p)
    assert rb.iterations == rs.iterations and np.array_equal(xb, xs)


def test_the_kernel_profile_reports_every_kernel():
    # dt_diff_profile_kernels on the benchmark's raster: a positive time and the algorithmic bytes
    w, h = 2048, 1024
    z0 = terrain(w, h, 17)
    kd = shelf_kd(z0, 17)
    ws = D.Workspace(D.Dims(w, h, 10_000.0, True))
    prof = ws.profile_kernels(kd, 1.0, reps=2)
    assert list(prof) == list(D.Workspace.PROFILE_KERNELS)
    n = w * h
    assert prof["apply_fp64"][1] == 40 * n and prof["apply_fp32"][1] == 20 * n
    assert all(t > 0 for t, _ in prof.values())
