"""The per-timestep elliptic solves in a loop: each step one flexure solve and then one implicit
diffusion solve on a w x h raster, with the load, rigidity and diffusivity fields re-seeded every
step (on the device), timed on the device.

    python deep-time_b200/timestep_loop.py --steps 100          # 16384 x 8192, dx 1.25 km

Per step:
  flexure   FP32 PCG with FP64 reliable updates, the reference's bank + Jacobi preconditioner,
            the U-Net's first guess (kept by the preconditioned-residual rule), to relative
            residual 1e-8; rigidity D = 10^(21 + 3u), u smoothed over --sigma cells; load
            2700 g h, h a |k|^-2 field of std 1500 m
  diffusion one FP32 CG on red-black Gauss-Seidel V(2,2) cycles with FP64 reliable updates (the
            residual replaced by the FP64 b - A x), to relative residual 1e-8; h a |k|^-2.5 field of std 800 m, kappa dt / dx^2 log-uniform
            over [0.1, 100] smoothed over --sigma cells
The plain FP64 path (mean-D preconditioner; FP64 CG and cycle) and the FP64 path with the
reference's preconditioner run --plain-steps steps each on the same seeds. With --cpu, the
oracle (the reference's CPU solvers restated, all host threads) solves the first step's fields
completely, to the same tolerance, timed by the wall clock. With --check, the first step's fast
and plain answers are compared with the oracle's FP64 solves (flexure PCG to relative residual
1e-12, diffusion's unpreconditioned CG to 1e-13): relative L2 and max-abs in metres.
"""
import argparse
import ctypes
import json
import os
import statistics
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--w", type=int, default=16384)
    ap.add_argument("--h", type=int, default=8192)
    ap.add_argument("--dx", type=float, default=1250.0)
    ap.add_argument("--sigma", type=float, default=64.0, help="smoothing of the rigidity and diffusivity fields, cells")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--plain-steps", type=int, default=3, help="steps of the plain FP64 path and of the FP64 bank path")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--dt", type=float, default=1.0, help="diffusion time step (kappa follows from kappa dt / dx^2)")
    ap.add_argument("--weights", default=os.path.join(HERE, "weights", "unet_flexure.bin"))
    ap.add_argument("--cpu", action="store_true", help="time the oracle's complete solves of the first step's fields")
    ap.add_argument("--check", action="store_true",
                    help="compare the first step's answers with the oracle's FP64 solves (rel-L2, max-abs)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()

    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import diffusion as Dm
    from deeptime_gpu import flexure as F
    from deeptime_gpu import unet as U

    lib = L.lib()
    dev = torch.device("cuda")
    w, h, dx = args.w, args.h, args.dx
    sv = F.Solver(w, h, dx)
    ws = Dm.Workspace(Dm.Dims(w, h, dx, True))
    model = None
    if os.path.exists(args.weights):
        model = U.UNet(seed=1)
        model.load(args.weights)
        L.check(lib.dt_flex_set_unet(sv._h, model._h, ctypes.c_double(10_000.0)))
    x = torch.zeros((h, w), dtype=torch.float64, device=dev)
    hd = torch.zeros((h, w), dtype=torch.float64, device=dev)

    fast_f = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_MIXED_RELIABLE,
                      warm_start=L.WARM_UNET if model else L.WARM_NONE, tol=args.tol, max_iterations=20000)
    plain_f = F.params(precond=L.PRECOND_MEAN_D, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_FP64, tol=args.tol,
                       max_iterations=20000)
    bank_f = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_FP64, tol=args.tol,
                      max_iterations=20000)
    fast_d = Dm.params(cycle=L.CYCLE_RBGS, precision=L.DIFF_MIXED_RELIABLE, stop=L.STOP_REL_RESIDUAL, tol=args.tol, max_iterations=2000)
    plain_d = Dm.params(cycle=L.CYCLE_RBGS, precision=L.DIFF_FP64, stop=L.STOP_REL_RESIDUAL, tol=args.tol, max_iterations=2000)

    def fields(step):
        d, c, b = U.flexure_problem_torch(w, h, args.sigma, 1000 + 2 * step, dev)
        h0, s = U.diffusion_problem_torch(w, h, args.sigma, 3000 + 2 * step, dev)
        return d, c, b, h0, s * dx * dx / args.dt

    def step_solves(step, pf, pd):
        d, c, b, h0, kd = fields(step)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rf = L.Report()
        L.check(lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                      ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()), ctypes.byref(pf),
                                      ctypes.byref(rf)))
        hd.copy_(h0)
        torch.cuda.synchronize()
        rd = L.Report()
        L.check(lib.dt_diff_solve_dev(ws._h, ctypes.c_void_p(hd.data_ptr()), ctypes.c_void_p(kd.data_ptr()),
                                      ctypes.c_double(args.dt), ctypes.byref(pd), ctypes.byref(rd)))
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        return {"flexure_ms": rf.device_ms, "flexure_iterations": rf.iterations, "flexure_rel_residual": rf.rel_residual,
                "warm_start_kept": bool(rf.warm_start_accepted), "diffusion_ms": rd.device_ms,
                "diffusion_iterations": rd.iterations, "diffusion_rel_residual": rd.rel_residual,
                "step_ms": rf.device_ms + rd.device_ms, "wall_ms": 1e3 * wall}

    # one untimed step per method first: graphs, level buffers and the model's buffers are made on
    # first use
    step_solves(0, fast_f, fast_d)
    fast = [step_solves(k, fast_f, fast_d) for k in range(args.steps)]
    step_solves(0, plain_f, plain_d)
    plain = [step_solves(k, plain_f, plain_d) for k in range(args.plain_steps)]
    step_solves(0, bank_f, plain_d)
    bank = [step_solves(k, bank_f, plain_d) for k in range(args.plain_steps)]

    def summary(rows):
        keys = ["step_ms", "wall_ms", "flexure_ms", "diffusion_ms", "flexure_iterations", "diffusion_iterations"]
        out = {k: statistics.mean(r[k] for r in rows) for k in keys}
        out["steps"] = len(rows)
        out["max_flexure_rel_residual"] = max(r["flexure_rel_residual"] for r in rows)
        out["max_diffusion_rel_residual"] = max(r["diffusion_rel_residual"] for r in rows)
        return out

    report = {"raster": f"{w}x{h}", "dx_m": dx, "sigma_cells": args.sigma, "tol": args.tol,
              "fast": summary(fast), "plain_fp64": summary(plain), "fp64_bank_fp64_diffusion": summary(bank),
              "warm_start_kept": sum(r["warm_start_kept"] for r in fast)}
    report["speedup_per_step"] = report["plain_fp64"]["step_ms"] / report["fast"]["step_ms"]

    if args.cpu or args.check:
        from oracle import oracle as O

        threads = O.set_threads(0)
        d, c, b, h0, kd = (t.cpu().numpy() for t in fields(0))
    if args.cpu:
        t = time.perf_counter()
        _, fr = O.flex_solve(d, c, b, dx, args.tol, 20000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
        tf = time.perf_counter() - t
        t = time.perf_counter()
        _, dit, _ = O.diff_solve_mg(h0, kd, args.dt, dx, args.tol, stop=O.STOP_REL_RESIDUAL, max_it=2000)
        td = time.perf_counter() - t
        cpu_ms = 1e3 * (tf + td)
        report["cpu_oracle"] = {"step_ms": cpu_ms, "threads": threads,
                                "how": f"the first step's fields solved completely to {args.tol:g}, wall clock: flexure "
                                       f"(FP64, the reference's bank + Jacobi) {tf:.1f} s in {fr['iterations']} "
                                       f"iterations, diffusion (FP64 CG, FP32 damped-Jacobi cycle) {td:.1f} s in "
                                       f"{dit} iterations"}
        report["speedup_vs_cpu"] = cpu_ms / report["fast"]["step_ms"]
    if args.check:
        want_x, _ = O.flex_solve(d, c, b, dx, 1e-12, 20000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
        want_h = O.diff_reference_cg(h0, kd, args.dt, dx, True, rel=1e-13)
        check = {"against": "the oracle's FP64 flexure PCG to relative residual 1e-12 and its diffusion CG to "
                            "1e-13, on the first step's fields"}
        for name, pf, pd in (("fast", fast_f, fast_d), ("plain_fp64", plain_f, plain_d)):
            step_solves(0, pf, pd)
            got_x, got_h = x.cpu().numpy(), hd.cpu().numpy()
            check[name] = {
                "flexure": {"rel_l2": float(np.linalg.norm(got_x - want_x) / np.linalg.norm(want_x)),
                            "max_abs_m": float(np.abs(got_x - want_x).max())},
                "diffusion": {"rel_l2": float(np.linalg.norm(got_h - want_h) / np.linalg.norm(want_h)),
                              "max_abs_m": float(np.abs(got_h - want_h).max())}}
        check["max_abs_deflection_m"] = float(np.abs(want_x).max())
        report["check"] = check
    print(json.dumps(report), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"report": report, "steps": fast, "plain_steps": plain, "bank_steps": bank}, f, indent=1)


if __name__ == "__main__":
    main()
