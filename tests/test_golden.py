"""The committed golden fixtures (tests/golden/, written by make_golden.py from the oracle) against
the generators and the oracle as they are now, on the CPU. A change to the input generators or to
the oracle's arithmetic shows up here first.

Tolerances: inputs bit-exact; operator outputs 1e-14 relative; preconditioners and solves 1e-10
relative (the oracle's OpenMP reductions may sum in another order).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import make_golden as G

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def flex():
    return np.load(os.path.join(HERE, "flexure_64x32.npz"))


@pytest.fixture(scope="module")
def diff():
    return np.load(os.path.join(HERE, "diffusion_64x32.npz"))


def test_the_generators_reproduce_the_fixture_inputs(flex, diff):
    d, c, b, v = G.flexure_inputs()
    for name, a in zip("dcbv", (d, c, b, v)):
        assert np.array_equal(a, flex[name]), name
    h0, kd = G.diffusion_inputs()
    assert np.array_equal(h0, diff["h0"]) and np.array_equal(kd, diff["kd"])


def test_the_oracle_reproduces_the_flexure_fixture(flex):
    out = G.flexure_outputs(flex["d"], flex["c"], flex["b"], flex["v"])
    for k in ("y_operator", "y_bend"):
        assert rel(out[k], flex[k]) <= 1e-14, k
    for k in ("z_mean_d", "z_reference", "x_reference_rule", "x_rel_1e-12"):
        assert rel(out[k], flex[k]) <= 1e-10, k
    assert out["iterations_reference_rule"] == flex["iterations_reference_rule"]


def test_the_oracle_reproduces_the_diffusion_fixture(diff):
    out = G.diffusion_outputs(diff["h0"], diff["kd"])
    assert rel(out["y_operator"], diff["y_operator"]) <= 1e-14
    for k in ("h_reference_rule", "h_rel_1e-12"):
        assert rel(out[k], diff[k]) <= 1e-10, k
    assert out["iterations_reference_rule"] == diff["iterations_reference_rule"]
