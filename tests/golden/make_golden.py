"""Writes the golden fixtures of this folder from the oracle (the CPU restatement of the
reference's solvers) on seeded inputs of the benchmark's generators:

    python tests/golden/make_golden.py

flexure_64x32.npz   inputs d, c, b (flexure_problem(64, 32, sigma 8, seed 1000)), v (SplitMix64
                    normal, seed 1001, x 50 m), dx = 10 km; outputs: the operator and bend of v,
                    the mean-D and reference preconditioners of b, the reference solve (max|z| <
                    2 m, 60 iterations: its x and iterations) and the reference-preconditioned
                    solve to relative residual 1e-12.
diffusion_64x32.npz inputs h0 and kd (diffusion_problem(64, 32, sigma 4, seed 2000), kd such that
                    kd dt / dx^2 = s), dt = 1000 yr, dx = 10 km; outputs: the operator of h0, the
                    reference multigrid solve (RMS 1e-5 m: h' and iterations) and the solve to
                    relative residual 1e-12.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "deep-time_b200"))

from oracle import oracle as O  # noqa: E402
from deeptime_gpu import inputs as I  # noqa: E402

FLEX = dict(w=64, h=32, dx=10_000.0, sigma=8.0, seed=1000)
DIFF = dict(w=64, h=32, dx=10_000.0, dt=1000.0, sigma=4.0, seed=2000)


def flexure_inputs():
    w, h = FLEX["w"], FLEX["h"]
    d, c, b = I.flexure_problem(w, h, FLEX["sigma"], FLEX["seed"])
    v = I.splitmix64_normal(FLEX["seed"] + 1, w * h).reshape(h, w) * 50.0
    return d, c, b, v


def diffusion_inputs():
    w, h, dx, dt = DIFF["w"], DIFF["h"], DIFF["dx"], DIFF["dt"]
    h0, s = I.diffusion_problem(w, h, DIFF["sigma"], DIFF["seed"])
    return h0, s * dx * dx / dt


def flexure_outputs(d, c, b, v):
    dx = FLEX["dx"]
    out = {
        "y_operator": O.flex_operator(d, c, v, dx),
        "y_bend": O.flex_bend(d, v, dx),
        "z_mean_d": O.flex_precondition(d, c, b, dx, precond=O.PRECOND_MEAN_D),
        "z_reference": O.flex_precondition(d, c, b, dx, precond=O.PRECOND_REFERENCE),
    }
    x, rep = O.flex_solve(d, c, b, dx, 2.0, 60)
    out["x_reference_rule"], out["iterations_reference_rule"] = x, np.int64(rep["iterations"])
    x, rep = O.flex_solve(d, c, b, dx, 1e-12, 5000, stop=O.STOP_REL_RESIDUAL)
    out["x_rel_1e-12"] = x
    return out


def diffusion_outputs(h0, kd):
    dx, dt = DIFF["dx"], DIFF["dt"]
    out = {"y_operator": O.diff_operator(h0, kd, dt, dx)}
    x, its, _ = O.diff_solve_mg(h0, kd, dt, dx, 1e-5)
    out["h_reference_rule"], out["iterations_reference_rule"] = x, np.int64(its)
    x, _, rel = O.diff_solve_mg(h0, kd, dt, dx, 1e-12, stop=O.STOP_REL_RESIDUAL, precision=64)
    out["h_rel_1e-12"] = x
    return out


def main():
    O.build()
    d, c, b, v = flexure_inputs()
    np.savez_compressed(os.path.join(HERE, "flexure_64x32.npz"), d=d, c=c, b=b, v=v, **flexure_outputs(d, c, b, v))
    h0, kd = diffusion_inputs()
    np.savez_compressed(os.path.join(HERE, "diffusion_64x32.npz"), h0=h0, kd=kd, **diffusion_outputs(h0, kd))


if __name__ == "__main__":
    main()
