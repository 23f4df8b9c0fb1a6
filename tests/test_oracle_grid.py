"""The oracle's restatement of the step's grid helpers around the flexure solve, pinned by the
reference's own tests of them (flexure.rs:4747-4761, grid.rs:286-392)."""
import numpy as np

from oracle import oracle as O


def test_restrict_and_the_constant_prolongation():
    # flexure.rs:4753-4758
    v = np.arange(64, dtype=np.float64).reshape(8, 8)
    r = O.restrict_by(v, 2)
    assert r.shape == (4, 4)
    assert r[0, 0] == (0.0 + 1.0 + 8.0 + 9.0) / 4.0
    assert np.array_equal(O.restrict_by(O.prolong_const(r, 2), 2), r)
    assert np.array_equal(O.restrict_by(v, 1), v)


def test_the_linear_prolongation_keeps_the_mean_and_constants():
    # flexure.rs:4759-4761
    v = np.arange(64, dtype=np.float64).reshape(8, 8)
    r = O.restrict_by(v, 2)
    lin = O.prolong_linear(r, 2)
    assert lin.shape == (8, 8)
    assert abs(lin.mean() - r.mean()) < 0.5
    assert np.array_equal(O.prolong_linear(r, 1), r)
    c = np.full((5, 6), 3.25)
    assert np.array_equal(O.prolong_linear(c, 4), np.full((20, 24), 3.25))


def test_the_linear_prolongation_interpolates_between_centres():
    # cell centres of the fine raster at (i + 0.5) / f - 0.5 in coarse units; x wraps
    ws, hs, f = 4, 3, 2
    v = np.arange(ws * hs, dtype=np.float64).reshape(hs, ws)
    lin = O.prolong_linear(v, f)
    # fine (i = 1, j = 1): x = y = 0.25 between coarse (0, 0), (1, 0), (0, 1), (1, 1)
    x = y = 0.25
    want = (v[0, 0] * (1 - x) + v[0, 1] * x) * (1 - y) + (v[1, 0] * (1 - x) + v[1, 1] * x) * y
    assert lin[1, 1] == want
    # fine i = 0: x = -0.25 wraps to the last coarse column
    x = 0.75
    want = (v[0, 3] * (1 - x) + v[0, 0] * x)
    assert lin[0, 0] == want


def test_the_binomial_filter():
    rng = np.random.default_rng(3)
    v = rng.standard_normal((16, 24))
    assert np.array_equal(O.binomial(v, 0), v)
    assert np.allclose(O.binomial(np.full((7, 9), 2.0), 3), 2.0, rtol=0, atol=0)
    # one pass by hand: x (wrapping) then y (rows clamped)
    t = 0.25 * np.roll(v, 1, axis=1) + 0.5 * v + 0.25 * np.roll(v, -1, axis=1)
    n = np.vstack([t[:1], t[:-1]])
    s = np.vstack([t[1:], t[-1:]])
    assert np.array_equal(O.binomial(v, 1), 0.25 * n + 0.5 * t + 0.25 * s)


def test_the_blur_keeps_the_mean_on_a_wrapping_band():
    # grid.rs:383-391
    c = np.arange(32 * 16)
    v = ((c * 7919) % 13).astype(np.float64).reshape(16, 32)
    before = v.sum()
    after = O.box_blur(v, 3, 3, wrap=True).sum()
    assert abs(before - after) < 1e-9 * before
