"""The device path through the C ABI against the committed golden fixtures (tests/golden/), which
need neither the oracle nor the reference at run time.

Tolerances: operators 1e-13 relative (FP64, another order of operations); the mean-D
preconditioner 1e-12 and the bank's 1e-8 (its sqrt(f) weights amplify ulp differences of log/pow
where f is tiny); solves to relative residual 1e-12 within 1e-8 relative L2 of the fixture (the
bar of the path); the reference's max|z| rule in the same number of iterations (one more or fewer
when the last max|z| sits at the threshold) and within 1e-8 relative L2 when the count agrees.
Diffusion: the cycle runs in FP32 on both sides, so the reference-rule solve is compared within
its RMS tolerance of 1e-5 m.
"""
import os

import numpy as np
import pytest

from deeptime_gpu import _lib as L
from deeptime_gpu import diffusion as D
from deeptime_gpu import flexure as F

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def flex():
    return np.load(os.path.join(HERE, "flexure_64x32.npz"))


@pytest.fixture(scope="module")
def diff():
    return np.load(os.path.join(HERE, "diffusion_64x32.npz"))


def test_flexure_operator_bend_and_preconditioners(flex):
    d, c, b, v = flex["d"], flex["c"], flex["b"], flex["v"]
    sv = F.Solver(64, 32, 10_000.0)
    assert rel(sv.operator(d, c, v), flex["y_operator"]) <= 1e-13
    assert rel(sv.bend(d, v), flex["y_bend"]) <= 1e-13
    assert rel(sv.precondition(d, c, b, precond=L.PRECOND_MEAN_D), flex["z_mean_d"]) <= 1e-12
    assert rel(sv.precondition(d, c, b, precond=L.PRECOND_REFERENCE), flex["z_reference"]) <= 1e-8


def test_flexure_solves(flex):
    d, c, b = flex["d"], flex["c"], flex["b"]
    sv = F.Solver(64, 32, 10_000.0)
    x, rep = sv.solve(d, c, b, 2.0, 60)
    assert abs(rep.iterations - int(flex["iterations_reference_rule"])) <= 1
    if rep.iterations == int(flex["iterations_reference_rule"]):
        assert rel(x, flex["x_reference_rule"]) <= 1e-8
    for precision in (L.PREC_FP64, L.PREC_MIXED, L.PREC_MIXED_RELIABLE):
        p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=precision, tol=1e-12,
                     max_iterations=5000)
        x, rep = sv.solve_with(d, c, b, p)
        assert rep.converged and rel(x, flex["x_rel_1e-12"]) <= 1e-8, (precision, rep)


def test_diffusion_operator_and_solves(diff):
    h0, kd = diff["h0"], diff["kd"]
    ws = D.Workspace(D.Dims(64, 32, 10_000.0, True))
    assert rel(ws.operator(kd, 1000.0, h0), diff["y_operator"]) <= 1e-13
    x, rep = ws.solve_with(h0, kd, 1000.0, D.params(tol=1e-5))
    assert abs(rep.iterations - int(diff["iterations_reference_rule"])) <= 1
    assert np.sqrt(np.mean((x.reshape(h0.shape) - diff["h_reference_rule"]) ** 2)) <= 1e-5
    for precision in (L.DIFF_FP64, L.DIFF_MIXED, L.DIFF_MIXED_RELIABLE):
        p = D.params(precision=precision, stop=L.STOP_REL_RESIDUAL, tol=1e-12)
        x, rep = ws.solve_with(h0, kd, 1000.0, p)
        assert rep.converged and rel(x.reshape(h0.shape), diff["h_rel_1e-12"]) <= 1e-8, (precision, rep)
