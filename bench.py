"""Benchmark: flexure solves per second to a relative residual of 1e-8 on a 4096 x 2048 raster.

Workload (the mixed-precision configuration): dx = 2.5 km, rigidity D = 10^(21 + 3u) with u
seeded white noise Gaussian-smoothed over 32 cells and rescaled to [0, 1], load q = 2700 g h with
h a seeded |k|^-2 Gaussian random field of std 1500 m, restoring density 3300 kg/m^3; PCG from
x = 0 (or the U-Net's first guess) to ||b - A x|| / ||b|| <= 1e-8. A step is one solve of one
input set; input sets are generated up front and cycled, each vector 67 MB, so the working set
(several hundred MB) is larger than the 126 MB L2 and no flush is needed between steps.

One process per GPU (torchrun for N > 1). The solves are independent, so N GPUs run N replicas
(weak scaling, no collective on the data path); rank 0 prints one JSON line with the whole-job
throughput over the max-over-ranks device time.

  value     solves/s with inputs resident in HBM (dt_flex_solve_dev, CUDA events, barrier and
            synchronize on both sides)
  e2e       the same through dt_flex_solve from pinned host buffers: the H2D copy of d, c, b and
            the D2H copy of x are inside the timed region
  roofline  the dominant kernel's algorithmic bytes per launch / its event-timed launch duration
  cpu_baseline  the oracle (a C++ restatement of the reference's CPU solver, FP64, its own
            3-level bank preconditioner) on the host's cores: complete solves to 1e-8 timed by
            the wall clock, on all host threads and on 8 (the reference's own bench setting)
  sphere    the same solve on the sphere's row metric (a band of latitudes +-58 degrees)
  step_raster  the timestep's own call at 1024 x 328 (39 km cells, max|z| < 2 m, at most 60
            iterations), FP64, device and end to end; the oracle's time for the same
            call sits in cpu_baseline
  grid_helpers  the step's restrict / prolong / binomial / box blur on an 8192 x 4096 raster,
            each call's bandwidth over its algorithmic bytes
  cube      the cube grid's diffusion at 6 x 256^2 cells, device and end to end; the oracle's
            time beside it in cpu_baseline
--impl reference times that CPU restatement alone, as the reference arm: complete solves of the
same input sets, one per step, after the warm-up solves.

Run as `python bench.py --gpus N` without torchrun's environment, it launches its own N ranks
(torch.distributed.run on 127.0.0.1) and rank 0 prints the line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "deep-time_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

W, H, DX, SIGMA = 4096, 2048, 2500.0, 32.0
TOL = 1e-8
REF_THREADS = 8  # the reference's own benchmark runs its solver pool on 8 threads
KERNEL_NAMES = ["flex_apply", "cg_update", "cg_direction", "fft_rows_fwd", "dct_cols_divide_idct", "fft_rows_inv_dot",
                "jacobi_left", "jacobi_final", "fft_rows_fwd_weighted", "fft_rows_inv_bank", "dct_cols_divide_idct_one_level"]
WEIGHTS = os.path.join(ROOT, "deep-time_b200", "weights", "unet_flexure.bin")
MODEL_DX = 10_000.0  # the U-Net's cell size: trained on 512 x 256 rasters of 10 km
METRIC = "flexure solves/s to relative residual 1e-8 @4096x2048 (time-to-1e-8 per solve = 1000/value ms)"


def set_raster(spec):
    """--raster W,H,DX_M,SIGMA: another raster for a quick check (the default is the 4096 x 2048 workload)."""
    global W, H, DX, SIGMA, METRIC
    w, h, dx, sg = spec.split(",")
    W, H, DX, SIGMA = int(w), int(h), float(dx), float(sg)
    METRIC = f"flexure solves/s to relative residual 1e-8 @{W}x{H} (time-to-1e-8 per solve = 1000/value ms)"


def workload_config(n_inputs):
    """The `config` both arms print: the workload alone, so that the two lines compare like for like."""
    return {"workload": f"flexure PCG to rel. residual {TOL:g}, {W}x{H}, dx {DX / 1e3:g} km, sigma {SIGMA:g} cells",
            "inputs": f"{n_inputs} seeded input sets cycled, {3 * W * H * 8 / 1e6:.0f} MB each: " +
                      ("larger than L2, no flush" if 3 * W * H * 8 > 126e6 else "smaller than L2 (a quick check)")}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--inputs", type=int, default=4, help="distinct seeded input sets cycled over the steps")
    ap.add_argument("--raster", default=None, help="W,H,DX_M,SIGMA: another flexure raster for a quick check")
    ap.add_argument("--precond", default="reference", choices=["reference", "mean_d"])
    ap.add_argument("--precision", default="reliable", choices=["reliable", "refinement"],
                    help="mixed precision of the benchmarked solve: one FP32 PCG with FP64 reliable updates, or FP32 "
                         "inner PCG inside FP64 iterative refinement (inner tolerance 1e-5)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the error against the oracle's 1e-12 solve")
    ap.add_argument("--no-diffusion", action="store_true", help="skip the diffusion solve's leg")
    ap.add_argument("--no-helpers", action="store_true",
                    help="skip the legs of the step's grid helpers and the cube grid's diffusion")
    ap.add_argument("--no-sphere", action="store_true", help="skip the sphere row metric's leg")
    ap.add_argument("--no-step-raster", action="store_true",
                    help="skip the timestep raster's leg (1024 x 328, the reference's max|z| rule)")
    ap.add_argument("--warm", default="unet" if os.path.exists(WEIGHTS) else "none", choices=["unet", "none"],
                    help="first guess of the benchmarked solve (default: the U-Net when trained weights exist)")
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--case", default=None,
                    help="profiling aid (for ncu): run one host-driven, iteration-capped solve and exit; "
                         "'W,H,DX,PRECOND,PRECISION,ITERATIONS' with PRECOND 0 reference / 1 mean-D and PRECISION "
                         "0 fp64 / 1 FP32 inside FP64 refinement / 2 FP32 with FP64 reliable updates")
    ap.add_argument("--diff-case", default=None,
                    help="profiling aid (for ncu): run one host-driven diffusion solve of the 2048 x 1024 workload's "
                         "recipe (red-black V(2,2), relative residual 1e-10) and exit; 'W,H,PRECISION' with PRECISION "
                         "0 the reference's split / 1 fp64 / 2 FP32 inside FP64 refinement / 3 FP32 with FP64 "
                         "reliable updates")
    return ap.parse_args()


def run_case(spec):
    from deeptime_gpu import _lib as L
    from deeptime_gpu import flexure as F
    from deeptime_gpu import inputs as I

    w, h, dx, pc, prec, its = spec.split(",")
    w, h, dx, pc, prec, its = int(w), int(h), float(dx), int(pc), int(prec), int(its)
    d, c, b = I.flexure_problem(w, h, 32.0 if w >= 2048 else 8.0, 1000)
    sv = F.Solver(w, h, dx)
    p = F.params(precond=pc, stop=L.STOP_REL_RESIDUAL, precision=prec, tol=TOL, max_iterations=its, host_loop=1)
    x, rep = sv.solve_with(d, c, b, p)
    print(rep, flush=True)


def run_diff_case(spec):
    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import diffusion as D
    from deeptime_gpu import inputs as I

    w, h, prec = (int(v) for v in spec.split(","))
    dx, dt = 10_000.0, 1.0
    h0, s = I.diffusion_problem(w, h, 8.0, 3000)
    ws = D.Workspace(D.Dims(w, h, dx, True))
    x, kd = torch.from_numpy(h0).cuda(), torch.from_numpy(s * dx * dx / dt).cuda()
    cycle = L.CYCLE_JACOBI if prec == L.DIFF_FP64_CG_FP32_CYCLE else L.CYCLE_RBGS
    p = D.params(cycle=cycle, precision=prec, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=2000, host_loop=1)
    rep = L.Report()
    L.check(L.lib().dt_diff_solve_dev(ws._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(kd.data_ptr()),
                                      ctypes.c_double(dt), ctypes.byref(p), ctypes.byref(rep)))
    print(f"iterations {rep.iterations}, converged {bool(rep.converged)}, relative residual {rep.rel_residual:.3e}, "
          f"refinements or replacements {rep.refinements}", flush=True)


def dist_init(n, timeout_s=300):
    """One process per GPU: NCCL when a device is present, gloo otherwise (the host logic's tests).
    The replicas exchange nothing but the barrier and the max over ranks of the timed region."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=timeout_s), device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=timedelta(seconds=timeout_s))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi samples (every 100 ms), started before the warm-up solves and stopped after the
    timed region; `wait_first` holds until the first sample has arrived, so the sampler is running
    when the timing starts."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def wait_first(self, timeout=5.0):
        t0 = time.perf_counter()
        while self.proc and not self.samples and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def make_inputs(k, seed0=1000):
    from deeptime_gpu import inputs as I

    return [I.flexure_problem(W, H, SIGMA, seed0 + 100 * i) for i in range(k)]


def oracle_full_solve_seconds(d, c, b):
    """Wall-clock seconds of one complete oracle solve to relative residual 1e-8 (FP64 PCG with the
    reference's 3-level bank + Jacobi preconditioner, from x = 0), and its iteration count."""
    from oracle import oracle as O

    t = time.perf_counter()
    _, rep = O.flex_solve(d, c, b, DX, TOL, 20000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
    return time.perf_counter() - t, rep["iterations"]


def oracle_cpu_baseline(inputs, solves=2):
    """The oracle's complete solves on the host: `solves` of them on all host threads (the median
    is the value) and one on 8 threads, each timed by the wall clock from x = 0 to 1e-8."""
    from oracle import oracle as O

    allc = O.set_threads(0)
    runs = [oracle_full_solve_seconds(*inputs[k % len(inputs)]) for k in range(solves)]
    secs = [r[0] for r in runs]
    t8 = O.set_threads(REF_THREADS)
    s8, it8 = oracle_full_solve_seconds(*inputs[0])
    O.set_threads(0)
    med = statistics.median(secs)
    return {"value": 1.0 / med, "unit": "solves/s", "cores": allc, "kind": "port",
            "sample": (f"{solves} complete solves of input sets 0..{solves - 1} to {TOL:g} by the oracle (FP64 PCG, the "
                       f"reference's 3-level bank + Jacobi preconditioner, x = 0), wall clock, OpenMP on all {allc} "
                       f"host threads; value = 1 / the median"),
            "seconds_per_solve": secs, "iterations": [r[1] for r in runs],
            "threads_8": {"value": 1.0 / s8, "seconds_per_solve": s8, "iterations": it8, "threads": t8,
                          "sample": "one complete solve of input set 0 on 8 host threads (the reference's bench setting)"}}


STEP_W, STEP_H, STEP_DX = 1024, 328, 39_000.0
STEP_TOL_M, STEP_MAX_IT = 2.0, 60


def step_inputs(k=2):
    from deeptime_gpu import inputs as I

    return [I.flexure_problem(STEP_W, STEP_H, 8.0, 5000 + 100 * i) for i in range(k)]


def oracle_step_seconds(sets):
    """The oracle's time per solve of the timestep raster's call (the reference preconditioner,
    max|z| < 2 m, at most 60 iterations), setup included, over the given input sets."""
    from oracle import oracle as O

    t = time.perf_counter()
    its = [O.flex_solve(d, c, b, STEP_DX, STEP_TOL_M, STEP_MAX_IT)[1]["iterations"] for d, c, b in sets]
    return (time.perf_counter() - t) / len(sets), its


def step_raster_leg(lib, stream, timed, max_over_ranks, world, steps, sets):
    """The timestep's own flexure call on its own raster: 1024 x 328 cells of 39 km (a height
    the cosine transform does not take, so y goes through the row solve with the block
    couplings), the reference preconditioner, max|z| < 2 m, at most 60 iterations, from x = 0.
    FP64, the reference's arithmetic (the mixed paths stop on residual rules only); device time
    per solve with inputs resident, and end to end through dt_flex_solve from pinned host
    buffers."""
    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import flexure as F

    sv = F.Solver(STEP_W, STEP_H, STEP_DX)
    L.check(lib.dt_flex_set_stream(sv._h, ctypes.c_void_p(stream.cuda_stream)))
    dev = [tuple(torch.from_numpy(a).cuda() for a in s) for s in sets]
    host = [tuple(torch.from_numpy(a).pin_memory() for a in s) for s in sets]
    x_dev = torch.zeros((STEP_H, STEP_W), dtype=torch.float64, device="cuda")
    x_host = torch.zeros((STEP_H, STEP_W), dtype=torch.float64).pin_memory()

    def call(fn, arrays, x, p):
        d, c, b = arrays
        rep = L.Report()
        L.check(fn(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                   ctypes.c_void_p(x.data_ptr()), ctypes.byref(p), ctypes.byref(rep)))
        return rep

    out = {"workload": f"flexure::step's solve, {STEP_W}x{STEP_H} at {STEP_DX / 1e3:g} km, reference 3-level bank + "
                       f"Jacobi, max|z| < {STEP_TOL_M:g} m, at most {STEP_MAX_IT} iterations, x = 0",
           "inputs": f"{len(sets)} seeded input sets cycled (rigidity sigma 8 cells, |k|^-2 topography of std 1500 m)"}
    for name, prec in (("fp64", L.PREC_FP64),):
        p = F.params(precision=prec, tol=STEP_TOL_M, max_iterations=STEP_MAX_IT)
        call(lib.dt_flex_solve_dev, dev[0], x_dev, p)
        ms, reps = timed(lambda i: call(lib.dt_flex_solve_dev, dev[i % len(dev)], x_dev, p), steps)
        ms = max_over_ranks(ms, world) / steps
        call(lib.dt_flex_solve, host[0], x_host, p)
        ems, _ = timed(lambda i: call(lib.dt_flex_solve, host[i % len(host)], x_host, p), steps)
        ems = max_over_ranks(ems, world) / steps
        out[name] = {"ms_per_solve": ms, "e2e_ms_per_solve": ems,
                     "iterations": statistics.mean(r.iterations for r in reps),
                     "converged": all(r.converged for r in reps),
                     "max_error_m": max(r.error_m for r in reps)}
    sv.close()
    return out


SPHERE_SIN = 0.85  # the band's edge: sin(58.2 degrees)


def sphere_leg(lib, stream, timed, max_over_ranks, world, steps, dev, fp, precond):
    """The headline's solve on the sphere's row metric (RowMetric::from_sin_faces, Solver::with_metric):
    the same 4096 x 2048 inputs, rows of equal area between latitudes +-58.2 degrees (sines of
    latitude at the row faces from 0.85 to -0.85), to relative residual 1e-8 with the reference
    preconditioner, FP64 and FP32 with FP64 reliable updates, from x = 0. The operator takes the
    rows' couplings and the spectral pass solves each wavenumber's pentadiagonal system along y."""
    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import flexure as F

    r_m = 0.5 * H * DX / SPHERE_SIN
    faces = np.clip((0.5 * H - np.arange(H + 1)) * DX / r_m, -1.0, 1.0)
    sv = F.Solver(W, H, DX, F.row_metric_from_sin_faces(faces))
    L.check(lib.dt_flex_set_stream(sv._h, ctypes.c_void_p(stream.cuda_stream)))
    x = torch.zeros((H, W), dtype=torch.float64, device="cuda")

    def solve(i, p):
        d, c, b = dev[i % len(dev)]
        rep = L.Report()
        L.check(lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                      ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()), ctypes.byref(p),
                                      ctypes.byref(rep)))
        return rep

    out = {"workload": f"the headline's {W}x{H} solve on the row metric, equal-area rows between sin(latitude) "
                       f"+-{SPHERE_SIN}, rel. residual {TOL:g}, reference preconditioner, x = 0"}
    for name, prec in (("fp64", L.PREC_FP64), ("mixed_reliable", L.PREC_MIXED_RELIABLE)):
        p = fp(prec, precond)
        solve(0, p)
        ms, reps = timed(lambda i: solve(i, p), steps)
        out[name] = {"ms_per_solve": max_over_ranks(ms, world) / steps,
                     "iterations": statistics.mean(r.iterations for r in reps),
                     "rel_residual": max(r.rel_residual for r in reps)}
    sv.close()
    return out


GRID_W, GRID_H = 8192, 4096
CUBE_N, CUBE_TOL_M, CUBE_DTS = 256, 1e-6, (7.0, 60.0)


def grid_leg(lib, stream, timed, max_over_ranks, world, steps, peak):
    """The step's grid helpers on a device raster of 8192 x 4096 FP64 cells (268 MB, larger than
    L2): the time per call and its bandwidth over the algorithmic bytes, each sweep reading and
    writing the raster once (restrict and prolongation read one raster and write the other)."""
    import torch

    from deeptime_gpu import _lib as L

    w, h, cells = GRID_W, GRID_H, GRID_W * GRID_H
    rng = np.random.default_rng(17)
    fine = torch.from_numpy(rng.standard_normal((h, w))).cuda()
    other = torch.empty_like(fine)
    coarse = torch.empty((h // 2, w // 2), dtype=torch.float64, device="cuda")
    sp = ctypes.c_void_p(stream.cuda_stream)

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    cases = {
        "restrict_by_2": (lambda: lib.dt_grid_restrict_dev(w, h, 2, P(fine), P(coarse), sp), 8 * cells * 1.25),
        "prolong_linear_2": (lambda: lib.dt_grid_prolong_linear_dev(w // 2, h // 2, 2, P(coarse), P(other), sp),
                             8 * cells * 1.25),
        "prolong_const_2": (lambda: lib.dt_grid_prolong_const_dev(w // 2, h // 2, 2, P(coarse), P(other), sp),
                            8 * cells * 1.25),
        "binomial_1_pass": (lambda: lib.dt_grid_binomial_dev(w, h, 1, P(fine), P(other), sp), 2 * 16 * cells),
        "box_blur_r2_2_passes": (lambda: lib.dt_grid_box_blur_dev(w, h, 1, 2, 2, P(fine), P(other), sp), 4 * 16 * cells),
    }
    out = {"raster": f"{w}x{h} FP64 ({8 * cells / 1e6:.0f} MB), the time per call, L2 not flushed (the raster is larger)"}
    for name, (fn, nbytes) in cases.items():
        L.check(fn())
        ms, _ = timed(lambda i: L.check(fn()), steps)
        ms = max_over_ranks(ms, world) / steps
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "algorithmic_bytes": nbytes, "GB/s": gbs, "frac_of_hbm_peak": gbs / peak}
    return out


def cube_leg(lib, stream, timed, max_over_ranks, world, steps, problem):
    """The cube grid's implicit diffusion (surface/cube/diffusion.rs::solve, the multigrid
    solver): 6 x 256^2 = 393 216 cells, the package's seeded geometry (cube.topology and
    inputs.cube_problem), RMS tolerance 1e-6 m, dt 7 and 60. Device time per solve with the
    fields resident (each step restores h on the stream first, 3 MB), and end to end through
    dt_cube_diff_solve from host arrays."""
    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import cube as C

    slots, lap, areas, kd, h0 = problem
    cd = C.CubeDiffusion(CUBE_N, slots, lap, areas)
    L.check(lib.dt_cube_set_stream(cd._h, ctypes.c_void_p(stream.cuda_stream)))
    kd_d, h0_d = torch.from_numpy(kd).cuda(), torch.from_numpy(h0).cuda()
    x_d = torch.empty_like(h0_d)
    x_h = [torch.from_numpy(h0.copy()).pin_memory() for _ in range(steps + 1)]

    def dev(dt):
        with torch.cuda.stream(stream):
            x_d.copy_(h0_d)
        rep = L.Report()
        L.check(lib.dt_cube_diff_solve_dev(cd._h, ctypes.c_void_p(x_d.data_ptr()), ctypes.c_void_p(kd_d.data_ptr()),
                                           ctypes.c_double(dt), ctypes.c_double(CUBE_TOL_M), ctypes.byref(rep)))
        return rep

    def host(dt, k):
        # a fresh pinned copy of h per call: the solve overwrites h in place
        rep = L.Report()
        L.check(lib.dt_cube_diff_solve(cd._h, ctypes.c_void_p(x_h[k].data_ptr()), ctypes.c_void_p(kd.ctypes.data),
                                       ctypes.c_double(dt), ctypes.c_double(CUBE_TOL_M), ctypes.byref(rep)))
        return rep

    out = {"workload": f"cube-grid implicit diffusion, 6x{CUBE_N}^2 cells, FP64 CG + FP32 damped-Jacobi V-cycle, "
                       f"RMS tolerance {CUBE_TOL_M:g} m", "levels": cd.levels}
    for dt in CUBE_DTS:
        dev(dt)
        ms, reps = timed(lambda i: dev(dt), steps)
        for t in x_h:
            t.copy_(torch.from_numpy(h0))
        host(dt, steps)
        ems, _ = timed(lambda i: host(dt, i), steps)
        out[f"dt_{dt:g}"] = {"ms_per_solve": max_over_ranks(ms, world) / steps,
                             "e2e_ms_per_solve": max_over_ranks(ems, world) / steps,
                             "iterations": statistics.mean(r.iterations for r in reps),
                             "rms_residual_m": max(r.error_m for r in reps)}
    cd.close()
    return out


def cube_problem():
    from deeptime_gpu import cube as C
    from deeptime_gpu import inputs as I

    slots = C.topology(CUBE_N)
    return (slots,) + tuple(I.cube_problem(CUBE_N, 5, slots))


def oracle_cube_ms(problem):
    """The oracle's time per cube solve at each dt, one solve each."""
    from oracle import oracle as O

    slots, lap, areas, kd, h0 = problem
    out = {}
    for dt in CUBE_DTS:
        t = time.perf_counter()
        _, its = O.cube_diff_solve(CUBE_N, slots, lap, areas, kd, dt, CUBE_TOL_M, h0)
        out[f"dt_{dt:g}"] = {"ms_per_solve": (time.perf_counter() - t) * 1e3, "iterations": its}
    return out


def run_reference(args, rank, world):
    """The reference arm: the oracle (the C++/OpenMP restatement of the reference's flexure::Solver,
    FP64 with its 3-level bank + Jacobi preconditioner) on all host threads, one complete solve to
    1e-8 from x = 0 per step over the same input sets as the device arm, after `warmup` untimed
    solves. Rank 0 alone runs it; the wall clock spans exactly the timed solves."""
    if rank != 0:
        return
    from oracle import oracle as O

    O.build() if not os.path.exists(O.LIB_PATH) else None
    cores = O.set_threads(0)
    inputs = make_inputs(max(1, args.inputs))
    for k in range(args.warmup):
        oracle_full_solve_seconds(*inputs[k % len(inputs)])
    secs, its = [], []
    t0 = time.perf_counter()
    for k in range(args.steps):
        s_k, i_k = oracle_full_solve_seconds(*inputs[k % len(inputs)])
        secs.append(s_k)
        its.append(i_k)
    total = time.perf_counter() - t0
    value = args.steps / total
    sample = (f"each step one complete solve of a {W}x{H} input set to {TOL:g} by the oracle (C++/OpenMP restatement of "
              f"the reference's flexure::Solver, FP64, 3-level bank + Jacobi, x = 0), wall clock, {cores} host threads; "
              f"{args.steps} timed solves in {total:.1f} s after {args.warmup} warm-up solves")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded SplitMix64 fields)",
            "impl": "reference", "config": workload_config(len(inputs)),
            "method": {"precision": "fp64", "preconditioner": "reference 3-level bank + Jacobi",
                       "iterations_per_solve": statistics.mean(its),
                       "seconds_per_solve": {"median": statistics.median(secs), "min": min(secs), "max": max(secs)}},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def launch_ranks(args):
    """`bench.py --gpus N` outside torchrun: run the same command as N local ranks under
    torch.distributed.run (127.0.0.1, a free port) and return its exit status."""
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.diff_case:
        run_diff_case(args.diff_case)
        return
    if args.case:
        run_case(args.case)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        raise SystemExit(launch_ranks(args))
    if args.raster:
        set_raster(args.raster)
    rank, world, local = dist_init(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import flexure as F

    torch.cuda.set_device(local)
    lib = L.lib()
    stream = torch.cuda.Stream()
    inputs = make_inputs(max(1, args.inputs), seed0=1000 + 7919 * rank)
    dev = [tuple(torch.from_numpy(a).cuda() for a in inp) for inp in inputs]
    x_dev = torch.zeros((H, W), dtype=torch.float64, device="cuda")
    sv = F.Solver(W, H, DX)
    L.check(lib.dt_flex_set_stream(sv._h, ctypes.c_void_p(stream.cuda_stream)))
    precond = L.PRECOND_REFERENCE if args.precond == "reference" else L.PRECOND_MEAN_D
    model = None
    if args.warm == "unet":
        if not os.path.exists(args.weights):
            raise SystemExit(f"--warm unet: no weights at {args.weights} (train them with deep-time_b200/train_unet.py)")
        from deeptime_gpu import unet as U

        model = U.UNet(seed=1)
        model.load(args.weights)
        L.check(lib.dt_flex_set_unet(sv._h, model._h, ctypes.c_double(MODEL_DX)))

    def fp(precision, pc, warm=L.WARM_NONE):
        return F.params(precond=pc, stop=L.STOP_REL_RESIDUAL, precision=precision, warm_start=warm, tol=TOL,
                        max_iterations=20000)

    head_prec = L.PREC_MIXED_RELIABLE if args.precision == "reliable" else L.PREC_MIXED
    head = fp(head_prec, precond, L.WARM_UNET if model else L.WARM_NONE)
    methods = {
        "plain_fp64_gpu": (fp(L.PREC_FP64, L.PRECOND_MEAN_D), "FP64 PCG, constant-mean-D spectral preconditioner"),
        "fp64_bank_gpu": (fp(L.PREC_FP64, L.PRECOND_REFERENCE), "FP64 PCG, reference 3-level bank + Jacobi"),
        "mixed_gpu": (fp(L.PREC_MIXED, precond), "FP32 inner PCG in FP64 refinement, zero first guess"),
        "mixed_reliable_gpu": (fp(L.PREC_MIXED_RELIABLE, precond), "FP32 PCG with FP64 reliable updates, zero first guess"),
    }

    def solve_dev(i, p):
        d, c, b = dev[i % len(dev)]
        rep = L.Report()
        st = lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                   ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x_dev.data_ptr()), ctypes.byref(p),
                                   ctypes.byref(rep))
        L.check(st)
        return rep

    def timed(fn, steps):
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps = [fn(i) for i in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return e0.elapsed_time(e1), reps

    with Clocks(local) as clk:
        for i in range(args.warmup):
            solve_dev(i, head)
        clk.wait_first()
        ms, reps = timed(lambda i: solve_dev(i, head), args.steps)
    ms = max_over_ranks(ms, world)
    its = [r.iterations for r in reps]
    launches = sum(r.kernel_launches for r in reps)
    head_ms = ms / args.steps

    # the other methods on the same inputs (the comparison the target names is plain_fp64_gpu)
    breakdown = {}
    for name, (p, what) in methods.items():
        solve_dev(0, p)
        k = min(args.steps, len(dev))
        pms, preps = timed(lambda i: solve_dev(i, p), k)
        pms = max_over_ranks(pms, world) / k
        breakdown[name] = {"ms_per_solve": pms, "iterations": statistics.mean(r.iterations for r in preps),
                           "method": what, "time_over_value": pms / head_ms}
    if model:
        breakdown["warm_start"] = {"accepted": sum(r.warm_start_accepted for r in reps), "of": len(reps),
                                   "mean_rel_preconditioned_residual": statistics.mean(r.warm_start_rel_residual
                                                                                       for r in reps)}

    # end to end through dt_flex_solve from pinned host buffers
    host = []
    for d, c, b in inputs:
        hs = [torch.from_numpy(a).pin_memory() for a in (d, c, b)]
        host.append(hs)
    x_host = torch.zeros((H, W), dtype=torch.float64).pin_memory()

    def solve_host(i):
        d, c, b = host[i % len(host)]
        rep = L.Report()
        st = lib.dt_flex_solve(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                               ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x_host.data_ptr()), ctypes.byref(head),
                               ctypes.byref(rep))
        L.check(st)
        return rep

    solve_host(0)
    e2e_steps = args.steps
    ems, _ = timed(solve_host, e2e_steps)
    ems = max_over_ranks(ems, world)

    # per-kernel launch durations (events) for the roofline
    kms = (ctypes.c_double * len(KERNEL_NAMES))()
    kbytes = (ctypes.c_double * len(KERNEL_NAMES))()
    solve_dev(0, methods["mixed_gpu"][0])
    L.check(lib.dt_flex_profile_kernels(sv._h, L.PREC_MIXED, 20, kms, kbytes))
    levels3 = args.precond == "reference"
    # the bank's column and weighted forward row passes: three launches an iteration, or one of the
    # three levels (the profile then reports three levels' bytes: 8 bytes a cell a level in the
    # FP32 lane); the mean-D preconditioner's one column pass is kernel 10
    bank = 3 // max(1, round(kbytes[4] / (2 * 4 * W * H)))
    per_it = ({0: 1, 1: 1, 2: 1, 6: 1, 7: 1, 8: bank, 4: bank, 9: 1} if levels3 else {0: 1, 1: 1, 2: 1, 3: 1, 10: 1, 5: 1})
    share = {k: kms[k] * cnt for k, cnt in per_it.items()}
    top = max(share, key=share.get)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else None
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    achieved = kbytes[top] / (kms[top] * 1e-3) / 1e9
    traffic = read_traffic(KERNEL_NAMES[top])
    kernels = {KERNEL_NAMES[k]: {"ms": kms[k], "GB/s": kbytes[k] / (kms[k] * 1e-3) / 1e9, "launches_per_iteration": cnt}
               for k, cnt in per_it.items()}

    value = world * args.steps / (ms / 1e3)
    warm_txt = "U-Net first guess (kept when its preconditioned residual is below the zero guess's)" if model \
        else "zero first guess"
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 inner / f64 refinement", "data": "synthetic (seeded SplitMix64 fields)",
        "config": workload_config(len(inputs)),
        "method": {"solve": ("mixed precision (one FP32 PCG, FP64 reliable updates of x and r), " if args.precision == "reliable"
                             else "mixed precision (FP32 inner PCG in FP64 refinement), ") +
                            f"{'reference 3-level bank + Jacobi' if levels3 else 'mean-D'} preconditioner, {warm_txt}",
                   "iterations_per_solve": statistics.mean(its), "replicas": world},
        "plain_fp64_gpu": dict(breakdown["plain_fp64_gpu"], speedup_of_value=breakdown["plain_fp64_gpu"]["ms_per_solve"] / head_ms),
        "methods": breakdown,
        "e2e": {"value": world * e2e_steps / (ems / 1e3), "unit": "solves/s",
                "h2d_bytes_per_step": 3 * W * H * 8, "d2h_bytes_per_step": W * H * 8},
        "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[top], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured copy)" if peaks else "fallback",
                     "traffic": traffic, "algorithmic_bytes_per_launch": kbytes[top], "kernels": kernels},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    if not args.no_diffusion:
        line["diffusion"] = diffusion_leg(lib, stream, timed, max_over_ranks, world, min(args.steps, 4),
                                          check=rank == 0 and not args.no_accuracy)
    if not args.no_sphere:
        line["sphere"] = sphere_leg(lib, stream, timed, max_over_ranks, world, min(args.steps, 2), dev, fp, precond)
    cube_case = None
    if not args.no_helpers:
        line["grid_helpers"] = grid_leg(lib, stream, timed, max_over_ranks, world, min(args.steps, 4), peak)
        cube_case = cube_problem()
        line["cube"] = cube_leg(lib, stream, timed, max_over_ranks, world, min(args.steps, 4), cube_case)
    step_sets = None
    if not args.no_step_raster:
        step_sets = step_inputs()
        line["step_raster"] = step_raster_leg(lib, stream, timed, max_over_ranks, world, args.steps, step_sets)
    if rank == 0 and not args.no_accuracy:
        line["accuracy"] = accuracy(lambda p: (solve_dev(0, p), x_dev.cpu().numpy())[1], head, methods, inputs[0])
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = oracle_cpu_baseline(inputs)
        if step_sets is not None:
            secs, its = oracle_step_seconds(step_sets)
            line["cpu_baseline"]["step_raster"] = {
                "ms_per_solve": secs * 1e3, "iterations": its,
                "sample": f"the oracle's solve of the step raster's call on each of its {len(step_sets)} input sets, "
                          f"setup included, OpenMP on all {os.cpu_count()} host threads"}
        if cube_case is not None:
            line["cpu_baseline"]["cube"] = dict(oracle_cube_ms(cube_case), sample=(
                f"the oracle's cube solve, one at each dt, OpenMP on all {os.cpu_count()} host threads"))
    if rank == 0:
        print(json.dumps(line), flush=True)
    sv.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def diffusion_leg(lib, stream, timed, max_over_ranks, world, steps, check=True):
    """The implicit diffusion solve at 2048 x 1024 (periodic x, closed rows): h a |k|^-2.5 field of
    std 800 m, kappa dt / dx^2 a smoothed log-uniform field over [0.1, 100] (sigma 8 cells),
    red-black Gauss-Seidel V(2,2) cycles to 16 x 8, CG to relative residual 1e-10; FP64 against
    FP32 inner CG + cycle inside FP64 refinement, and the reference's own split (FP64 CG, FP32
    damped-Jacobi cycle). Device time per solve (inputs resident); with `check`, each answer's
    relative L2 and max-abs error against the oracle's unpreconditioned FP64 CG to 1e-13 on input
    set 0."""
    import torch

    from deeptime_gpu import _lib as L
    from deeptime_gpu import diffusion as D
    from deeptime_gpu import inputs as I

    w, h, dx, dt = 2048, 1024, 10_000.0, 1.0
    ws = D.Workspace(D.Dims(w, h, dx, True))
    L.check(lib.dt_diff_set_stream(ws._h, ctypes.c_void_p(stream.cuda_stream)))
    sets = [I.diffusion_problem(w, h, 8.0, 3000 + 100 * k) for k in range(2)]
    dev = [(torch.from_numpy(h0).cuda(), torch.from_numpy(s * dx * dx / dt).cuda()) for h0, s in sets]
    x = torch.empty_like(dev[0][0])

    def solve(i, p):
        h0, kd = dev[i % len(dev)]
        with torch.cuda.stream(stream):
            x.copy_(h0)
        rep = L.Report()
        L.check(lib.dt_diff_solve_dev(ws._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(kd.data_ptr()),
                                      ctypes.c_double(dt), ctypes.byref(p), ctypes.byref(rep)))
        return rep

    out = {"workload": f"implicit diffusion {w}x{h}, kappa dt/dx^2 log-uniform [0.1, 100], CG to rel. residual 1e-10"}
    answers = {}
    for name, cycle, prec in (("fp64_rbgs", L.CYCLE_RBGS, L.DIFF_FP64), ("mixed_rbgs", L.CYCLE_RBGS, L.DIFF_MIXED),
                              ("mixed_reliable_rbgs", L.CYCLE_RBGS, L.DIFF_MIXED_RELIABLE),
                              ("reference_split_jacobi", L.CYCLE_JACOBI, L.DIFF_FP64_CG_FP32_CYCLE)):
        p = D.params(cycle=cycle, precision=prec, stop=L.STOP_REL_RESIDUAL, tol=1e-10, max_iterations=2000)
        solve(0, p)
        ms, reps = timed(lambda i: solve(i, p), steps)
        ms = max_over_ranks(ms, world) / steps
        solve(0, p)
        torch.cuda.synchronize()
        answers[name] = x.clone()
        out[name] = {"ms_per_solve": ms, "solves_per_s": world * 1e3 / ms,
                     "iterations": statistics.mean(r.iterations for r in reps),
                     "rel_residual": max(r.rel_residual for r in reps)}
    if check:
        from oracle import oracle as O

        h0, s0 = sets[0]
        exact = O.diff_reference_cg(h0, s0 * dx * dx / dt, dt, dx, True, rel=1e-13)
        out["accuracy_against"] = "the oracle's unpreconditioned FP64 CG to relative residual 1e-13, input set 0"
        for name, x_dev in answers.items():
            got = x_dev.cpu().numpy()
            out[name]["rel_l2"] = float(np.linalg.norm(got - exact) / np.linalg.norm(exact))
            out[name]["max_abs_m"] = float(np.abs(got - exact).max())
    # the finest level's hot kernels, each launch alone after an L2 flush: bandwidth over their
    # algorithmic bytes, against the measured copy peak
    peaks = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks))["hbm_gbs"] if os.path.exists(peaks) else 6650.0
    def kernels(prof):
        return {name: {"ms": t, "algorithmic_bytes": by, "GB/s": by / (t * 1e-3) / 1e9,
                       "frac_of_hbm_peak": by / (t * 1e-3) / 1e9 / peak} for name, (t, by) in prof.items()}

    out["kernels"] = kernels(ws.profile_kernels(sets[0][1] * dx * dx / dt, dt))
    # the same kernels at 8192 x 4096, where a launch is long enough that its fixed costs (the
    # ramp of the grid, the last block's reduction) weigh little beside its bytes
    wl, hl = 8192, 4096
    big = D.Workspace(D.Dims(wl, hl, dx, True))
    _, sl = I.diffusion_problem(wl, hl, 8.0, 3000)
    out["kernels_8192x4096"] = kernels(big.profile_kernels(sl * dx * dx / dt, dt))
    big.close()
    out["speedup_mixed_vs_fp64"] = out["fp64_rbgs"]["ms_per_solve"] / out["mixed_rbgs"]["ms_per_solve"]
    out["speedup_mixed_reliable_vs_fp64"] = out["fp64_rbgs"]["ms_per_solve"] / out["mixed_reliable_rbgs"]["ms_per_solve"]
    ws.close()
    return out


def accuracy(solve_x, head, methods, inp):
    """Errors of the benchmarked solve (and the plain one) against the oracle's FP64 solve (the
    reference's preconditioner) to relative residual 1e-12, on the first input set."""
    from oracle import oracle as O

    d, c, b = inp
    t = time.perf_counter()
    xo, rep = O.flex_solve(d, c, b, DX, 1e-12, 5000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
    secs = time.perf_counter() - t
    out = {"against": f"oracle FP64 PCG (reference preconditioner) to rel. residual 1e-12 "
                      f"({rep['iterations']} iterations, {secs:.1f} s on the host), input set 0"}
    norm = float(np.linalg.norm(xo))
    for name, p in (("value", head), ("plain_fp64_gpu", methods["plain_fp64_gpu"][0])):
        x = solve_x(p)
        out[name] = {"rel_l2": float(np.linalg.norm(x - xo)) / norm, "max_abs_m": float(np.abs(x - xo).max())}
    out["max_abs_deflection_m"] = float(np.abs(xo).max())
    return out


def read_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if one was captured."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


if __name__ == "__main__":
    main()
