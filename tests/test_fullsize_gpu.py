"""The configurations at their full sizes against the FP64 oracle, and what the trained U-Net's
first guess gains.

- Diffusion, 2048 x 1024 (periodic x, closed rows; h a |k|^-2.5 field of std 800 m, kappa dt/dx^2
  a smoothed log-uniform field over [0.1, 100]): red-black Gauss-Seidel V(2,2) multigrid CG to
  relative residual 1e-10, FP64 and FP32-cycle/FP64-refinement, and the reference's own split
  (FP64 CG, FP32 damped-Jacobi cycle), against the oracle's unpreconditioned CG to 1e-13
  (multigrid/tests.rs:17-74's oracle), and one FP32 CG with FP64 reliable updates on the same
  cycle. Bound: relative L2 <= 1e-8, max-abs <= 1e-8 of max |h'|.
- Flexure, 4096 x 2048 (dx 2.5 km, rigidity smoothed over 32 cells): the benchmarked method (FP32
  PCG with FP64 reliable updates, the reference preconditioner, the U-Net's first guess when the
  trained weights are present) and the plain FP64 mean-D method to relative residual 1e-8,
  against the oracle's FP64 PCG to 1e-12. Bound: relative L2 <= 1e-8; max-abs in metres printed.
- The trained U-Net: held-out seeds the training never saw, solved to 1e-10 at 512 x 256 and to
  1e-8 at 4096 x 2048 with and without the first guess; the guess must be kept and must save
  iterations.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import _lib as L
from deeptime_gpu import diffusion as D
from deeptime_gpu import flexure as F
from deeptime_gpu import inputs as I

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "deep-time_b200", "weights", "unet_flexure.bin")
MODEL_DX = 10_000.0


def errors(x, ref):
    return float(np.linalg.norm(x - ref) / np.linalg.norm(ref)), float(np.abs(x - ref).max())


@pytest.fixture(scope="module")
def diffusion_case():
    w, h, dx, dt = 2048, 1024, 10_000.0, 1.0
    topo, s = I.diffusion_problem(w, h, 8.0, 3000)
    kd = s * dx * dx / dt  # kappa dt / dx^2 = s, faces the arithmetic means
    exact = O.diff_reference_cg(topo, kd, dt, dx, True, rel=1e-13)
    return w, h, dx, dt, topo, kd, exact


@pytest.mark.parametrize("name,cycle,precision", [("fp64_rbgs", L.CYCLE_RBGS, L.DIFF_FP64),
                                                  ("mixed_rbgs", L.CYCLE_RBGS, L.DIFF_MIXED),
                                                  ("mixed_reliable_rbgs", L.CYCLE_RBGS, L.DIFF_MIXED_RELIABLE),
                                                  ("reference_split", L.CYCLE_JACOBI, L.DIFF_FP64_CG_FP32_CYCLE)])
def test_the_diffusion_config_at_full_size_matches_the_oracle(diffusion_case, name, cycle, precision):
    w, h, dx, dt, topo, kd, exact = diffusion_case
    ws = D.Workspace(D.Dims(w, h, dx, True))
    x, rep = ws.solve_with(topo, kd, dt, D.params(cycle=cycle, precision=precision, stop=L.STOP_REL_RESIDUAL,
                                                  tol=1e-10, max_iterations=2000))
    rel, mx = errors(x, exact)
    print(f"diffusion 2048x1024 {name}: {rep.iterations} iterations, rel. residual {rep.rel_residual:.2e}, "
          f"rel-L2 {rel:.2e}, max-abs {mx:.2e} m")
    assert rep.converged and rep.rel_residual <= 1e-10, rep
    assert rel <= 1e-8
    assert mx <= 1e-8 * np.abs(exact).max()
    assert abs(x.sum() - topo.sum()) <= 1e-9 * np.abs(topo).sum()


@pytest.fixture(scope="module")
def flexure_case():
    w, h, dx = 4096, 2048, 2500.0
    d, c, b = I.flexure_problem(w, h, 32.0, 1000)
    xo, rep = O.flex_solve(d, c, b, dx, 1e-12, 5000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
    assert rep["converged"]
    return w, h, dx, d, c, b, xo


def solver_with_unet(w, h, dx):
    sv = F.Solver(w, h, dx)
    model = None
    if os.path.exists(WEIGHTS):
        from deeptime_gpu import unet as U

        model = U.UNet(seed=1)
        model.load(WEIGHTS)
        L.check(L.lib().dt_flex_set_unet(sv._h, model._h, ctypes.c_double(MODEL_DX)))
    return sv, model


def test_the_mixed_flexure_config_at_full_size_matches_the_oracle(flexure_case):
    w, h, dx, d, c, b, xo = flexure_case
    sv, model = solver_with_unet(w, h, dx)
    cases = {"benchmarked": F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_MIXED_RELIABLE,
                                     warm_start=L.WARM_UNET if model else L.WARM_NONE, tol=1e-8, max_iterations=20000),
             "refinement": F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_MIXED,
                                    tol=1e-8, max_iterations=20000),
             "plain_fp64": F.params(precond=L.PRECOND_MEAN_D, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_FP64, tol=1e-8,
                                    max_iterations=20000)}
    for name, p in cases.items():
        x, rep = sv.solve_with(d, c, b, p)
        rel, mx = errors(x, xo)
        print(f"flexure 4096x2048 {name}: {rep.iterations} iterations, rel. residual {rep.rel_residual:.2e}, "
              f"rel-L2 {rel:.2e}, max-abs {mx:.2e} m (max |w| {np.abs(xo).max():.0f} m)")
        assert rep.converged and rep.rel_residual <= 1e-8, (name, rep)
        assert rel <= 1e-8, name


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained weights")
@pytest.mark.parametrize("w,h,dx,sigma,tol,seeds", [
    (512, 256, 10_000.0, 8.0, 1e-10, [50_000 + 2 * k for k in range(18_000, 18_008)]),  # held out of training
    (4096, 2048, 2500.0, 32.0, 1e-8, [1000, 1100]),                                    # the benchmark's raster
])
def test_the_trained_unet_saves_iterations_on_held_out_seeds(w, h, dx, sigma, tol, seeds):
    import torch

    from deeptime_gpu import unet as U

    sv, model = solver_with_unet(w, h, dx)
    lib = L.lib()
    dev = torch.device("cuda")
    x = torch.zeros((h, w), dtype=torch.float64, device=dev)
    cold, warm = [], []
    for seed in seeds:
        d, c, b = U.flexure_problem_torch(w, h, sigma, seed, dev)
        torch.cuda.synchronize()
        for start, out in ((L.WARM_NONE, cold), (L.WARM_UNET, warm)):
            rep = L.Report()
            p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, tol=tol, max_iterations=20000,
                         warm_start=start)
            L.check(lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                          ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()), ctypes.byref(p),
                                          ctypes.byref(rep)))
            assert rep.converged and rep.rel_residual <= tol
            out.append((rep.iterations, rep.warm_start_accepted, rep.warm_start_rel_residual))
    its_cold = [c[0] for c in cold]
    its_warm = [c[0] for c in warm]
    print(f"{w}x{h} to {tol:g}: zero guess {its_cold}, U-Net guess {its_warm}, "
          f"guess residual / zero guess's {[round(c[2], 3) for c in warm]}")
    assert all(c[1] for c in warm), "the guess was discarded"
    assert all(c[2] < 0.5 for c in warm)
    assert sum(its_warm) < sum(its_cold)
    assert all(a <= b + 1 for a, b in zip(its_warm, its_cold))
