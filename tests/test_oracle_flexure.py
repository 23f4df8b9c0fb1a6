"""Pins the CPU oracle's flexure solve to the reference's own known-answer tests.

Each test restates one from crates/deeptime-core/src/surface/flexure.rs `mod tests` with the same
grids, loads and tolerances (line numbers cited per test). The reference has no golden binary
vectors for this path: these analytic checks (plate theory) are what pins it.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

G = 9.81
RHO_M = O.RHO_MANTLE
RHO_W = O.RHO_WATER


def uniform(shape, te_km, g=G):
    return np.full(shape, O.rigidity_per_g(te_km, g)), np.full(shape, RHO_M)


def test_transform_round_trip():
    # flexure.rs:2813-2828: forward then inverse is the identity on even and odd rasters.
    for tw, th in [(256, 128), (15, 9), (12, 7)]:
        c = np.arange(tw * th)
        v = ((c * 7919) % 101).astype(np.float64) - 50.0
        back = O.spectral_roundtrip(v.reshape(th, tw), 10_000.0)
        assert np.max(np.abs(back.ravel() - v)) < 1e-9, (tw, th)


def test_a_point_load_sinks_by_the_analytic_depth():
    # flexure.rs:2810-2853
    w, h, dx = 256, 128, 10_000.0
    d, c = uniform((h, w), 30.0)
    l = (d[0, 0] / RHO_M) ** 0.25
    assert l / dx > 4.0
    mass = 1.0e15
    b = np.zeros((h, w))
    b[h // 2, w // 2] = mass / (dx * dx)
    x, rep = O.flex_solve(d, c, b, dx, 1e-9, 50)
    assert rep["converged"] and rep["iterations"] <= 1, rep
    analytic = mass / (8.0 * RHO_M * l * l)
    assert abs(x[h // 2, w // 2] / analytic - 1.0) < 0.03
    displaced = x.sum() * RHO_M * dx * dx
    assert abs(displaced / mass - 1.0) < 1e-9
    lowest = x.min()
    assert lowest < 0.0 and lowest > -0.05 * analytic


def line_load(te_km, g, dx):
    # flexure.rs:2857-2886
    w, h = 16, 1024
    d, c = uniform((h, w), te_km, g)
    alpha = O.flexural_parameter_m(d[0, 0])
    per_m = 1.0e10
    row = h // 2
    b = np.zeros((h, w))
    b[row, :] = per_m / dx
    x, rep = O.flex_solve(d, c, b, dx, 1e-9, 50)
    assert rep["converged"], rep
    profile = x[row:, 0]
    w0 = profile[0]
    k = int(np.argmax(profile < 0.0))
    zero = (k - 1.0 + profile[k - 1] / (profile[k - 1] - profile[k])) * dx
    kb = int(np.argmin(profile))
    return w0, zero, kb * dx, profile[kb], per_m / (2.0 * RHO_M * alpha)


def test_a_line_load_gives_the_analytic_profile():
    # flexure.rs:2890-2931
    dx, te = 5000.0, 30.0
    alpha = O.flexural_parameter_m(O.rigidity_per_g(te, G))
    assert abs(alpha / 1000.0 - 67.0) < 2.0
    w0, zero, bulge_at, bulge, analytic = line_load(te, G, dx)
    assert abs(w0 / analytic - 1.0) < 0.01
    assert abs(zero / (0.75 * math.pi * alpha) - 1.0) < 0.02
    assert abs(bulge_at - math.pi * alpha) <= 1.5 * dx
    assert abs(bulge / w0 + math.exp(-math.pi)) < 0.003
    _, zero2, *_ = line_load(2.0 * te, G, dx)
    assert abs(zero2 / zero - 2.0 ** 0.75) < 0.02
    w0m, zerom, *_ = line_load(te, 3.71, dx)
    assert abs(zerom / zero - (G / 3.71) ** 0.25) < 0.02
    assert w0m < w0


def broken_line_load(te_km, soft_km, dx):
    # flexure.rs:2937-2963
    w, h = 16, 1024
    row = h // 2
    rows = np.arange(h)[:, None] * np.ones((1, w))
    d = np.where(rows >= row, O.rigidity_per_g(te_km, G), O.rigidity_per_g(soft_km, G))
    c = np.full((h, w), RHO_M)
    alpha = O.flexural_parameter_m(O.rigidity_per_g(te_km, G))
    per_m = 1.0e10
    b = np.zeros((h, w))
    b[row, :] = per_m / dx
    x, rep = O.flex_solve(d, c, b, dx, 1e-6, 400)
    assert rep["converged"], rep
    profile = x[row:, 0]
    k = int(np.argmax(profile < 0.0))
    zero = (k - 1.0 + profile[k - 1] / (profile[k - 1] - profile[k])) * dx
    kb = int(np.argmin(profile))
    stiff = profile.sum() * dx * RHO_M / per_m
    return profile[0], zero, kb * dx, profile[kb], alpha, stiff


def test_a_line_load_on_a_broken_plate_gives_the_analytic_profile():
    # flexure.rs:2976-3018
    te, soft = 30.0, 0.5

    def error(dx):
        w0, _, _, _, alpha, stiff = broken_line_load(te, soft, dx)
        return w0 / (2.0 * stiff * 1.0e10 / (RHO_M * alpha)) - 1.0

    coarse, fine = error(5000.0), error(2500.0)
    assert abs(fine) < 0.06
    assert abs(fine / coarse - 0.5) < 0.1
    dx = 2500.0
    w0, zero, bulge_at, bulge, alpha, stiff = broken_line_load(te, soft, dx)
    assert 0.85 < stiff <= 1.0
    assert abs(zero / (0.5 * math.pi * alpha) - 1.0) < 0.015
    assert abs(bulge_at - 0.75 * math.pi * alpha) <= 2.0 * dx
    want = math.exp(-0.75 * math.pi) * math.cos(0.75 * math.pi)
    assert abs(bulge / w0 - want) < 0.002
    c0, czero, *_ = line_load(te, G, dx)
    assert w0 > 3.0 * c0 and zero < 0.7 * czero


def patchy(w, h, lo, hi):
    # flexure.rs:3020-3036
    j, i = np.mgrid[0:h, 0:w]
    te = np.where(((i // 24) + (j // 24)) % 3 == 0, hi, lo).astype(np.float64)
    return O.box_blur(te, 2, 2, wrap=True)


def test_a_patchy_plate_converges_and_compensates():
    # flexure.rs:3039-3080
    w, h, dx = 192, 96, 39_000.0
    te = patchy(w, h, 6.0, 70.0)
    d = np.vectorize(lambda t: O.rigidity_per_g(t, G))(te)
    k = np.arange(w * h).reshape(h, w)
    c = np.where((k % w) < w // 3, RHO_M - RHO_W, RHO_M)
    i, j = k % w, k // w
    mask = ((i % 37 < 3) & (j % 29 < 9)) | ((i + 2 * j) % 61 == 0)
    b = np.where(mask, RHO_M * (500.0 + ((k * 31) % 17) * 250.0), 0.0)
    x, rep = O.flex_solve(d, c, b, dx, 0.01, 400)
    assert rep["converged"] and rep["iterations"] < 150, rep
    left = b - O.flex_operator(d, c, x, dx)
    node_d, c_ref, weights = O.flex_bank(d, c, dx)
    # spectral_solve of the bank alone (no sweeps): the bank's blend of exact solves
    more = bank_spectral_solve(d, c, left, dx)
    assert np.max(np.abs(more)) < 0.05
    assert abs((x * c).sum() / b.sum() - 1.0) < 1e-3
    airy_wet = RHO_M / (RHO_M - RHO_W)
    assert x.max() < 4500.0 * airy_wet


def bank_spectral_solve(d, c, r, dx):
    """The bank's blended spectral solve: sum_k w_k S_k (w_k r), from the oracle's round trip
    pieces (flexure.rs:1654-1675). Built from flex_precondition on a plate where the bank has one
    level, otherwise per level with weights."""
    node_d, c_ref, weights = O.flex_bank(d, c, dx)
    h, w = r.shape
    if weights is None:
        return O.flex_precondition(np.full_like(d, node_d[0]), np.full_like(c, c_ref), r, dx, precond=O.PRECOND_MEAN_D)
    z = np.zeros_like(r)
    for k in range(len(node_d)):
        part = O.flex_precondition(np.full_like(d, node_d[k]), np.full_like(c, c_ref), r * weights[k], dx,
                                   precond=O.PRECOND_MEAN_D)
        z += part * weights[k]
    return z


def test_the_solve_is_stable_at_the_editors_extremes():
    # flexure.rs:3146-3164
    w, h, dx = 128, 64, 39_000.0
    for lo, hi in [(1.25, 20.0), (15.0, 240.0), (0.1, 1.0), (300.0, 500.0)]:
        te = patchy(w, h, lo, hi)
        d = np.vectorize(lambda t: O.rigidity_per_g(t, G))(te)
        c = np.full((h, w), RHO_M)
        b = np.zeros(w * h)
        b[::53] = RHO_M * 3000.0
        b = b.reshape(h, w)
        x, rep = O.flex_solve(d, c, b, dx, 0.1, 400)
        assert rep["converged"], (lo, hi, rep)
        assert np.all(np.isfinite(x))
        ratio = x.sum() * RHO_M / b.sum()
        assert abs(ratio - 1.0) < 1e-3, (lo, hi, ratio)
        assert x.max() <= 3000.0 * 1.001


def sphere_faces(h, dx, r_m):
    # flexure.rs:5341-5345
    k = np.arange(h + 1)
    return np.clip((0.5 * h - k) * dx / r_m, -1.0, 1.0)


@pytest.mark.parametrize("h,f,r_frac", [(164, 1, 0.5), (41, 1, 0.3), (300, 2, 1.0), (2048, 1, 0.59)])
def test_the_packages_row_metric_is_the_oracles(h, f, r_frac):
    # the metric a caller builds with the package (deeptime_gpu.flexure.row_metric_from_sin_faces),
    # bit for bit, on rasters that reach the poles (r_frac <= 0.5) and bands that do not
    from deeptime_gpu import flexure as F

    dx = 10_000.0
    faces = sphere_faces(h * f, dx, r_frac * h * f * dx)
    a, b = F.row_metric_from_sin_faces(faces, f)
    ao, bo = O.row_metric_from_sin_faces(faces, f)
    assert np.array_equal(a, ao) and np.array_equal(b, bo)


def test_the_row_metric_is_the_block_metric_at_the_equator():
    # flexure.rs:5351-5381
    w, h = 512, 164
    r_m = 6.371e6
    dx = 2 * math.pi * r_m / w
    faces = sphere_faces(h, dx, r_m)
    assert faces[0] == 1.0 and faces[h] == -1.0
    a, b = O.row_metric_from_sin_faces(faces, 1)
    assert (len(a), len(b)) == (h, h + 1)
    assert b[0] == 0.0 and b[h] == 0.0
    assert b[h // 2] == 1.0
    assert abs(a[h // 2] - 1.0) < 1e-4
    for j in range(h):
        s = 0.5 * (faces[j] + faces[j + 1])
        if abs(s) < 0.99:
            assert abs(a[j] * (1.0 - s * s) - 1.0) < 1e-12
            assert abs(b[j + 1] - (1.0 - faces[j + 1] ** 2)) < 1e-15
        assert np.isfinite(a[j]) and a[j] >= 1.0
    a2, b2 = O.row_metric_from_sin_faces(faces, 2)
    assert (len(a2), len(b2)) == (h // 2, h // 2 + 1)
    assert b2[1] == 1.0 - faces[2] * faces[2]


def test_the_solve_on_the_sphere_inverts_its_operator():
    # flexure.rs:5388-5456
    w, h, dx = 64, 32, 50_000.0
    faces = sphere_faces(h, dx, 0.49 * h * dx)
    metric = O.row_metric_from_sin_faces(faces, 1)
    n = w * h
    cidx = np.arange(n)

    def noise(seed):
        return ((((cidx * 7919 + seed * 104_729) % 1009).astype(np.float64) - 504.0) * 10.0).reshape(h, w)

    d = np.where(((cidx // w) % 9) < 4, O.rigidity_per_g(40.0, G), O.rigidity_per_g(8.0, G)).reshape(h, w)
    cr = np.where(cidx % w < 20, RHO_M - RHO_W, RHO_M).reshape(h, w).astype(np.float64)
    u, v = noise(1), noise(2)
    au = O.flex_operator(d, cr, u, dx, metric)
    av = O.flex_operator(d, cr, v, dx, metric)
    uav, vau = float((u * av).sum()), float((v * au).sum())
    assert abs(uav - vau) <= 1e-12 * max(abs(uav), abs(vau))
    du, cu = uniform((h, w), 25.0)
    b = noise(3)
    x, rep = O.flex_solve(du, cu, b, dx, 1e-9, 20, metric=metric)
    assert rep["iterations"] == 1, rep
    ax = O.flex_operator(du, cu, x, dx, metric)
    top = np.abs(b).max()
    assert np.abs(ax - b).max() < 1e-9 * top
    block = (np.ones(h), np.array([0.0] + [1.0] * (h - 1) + [0.0]))
    xr, _ = O.flex_solve(du, cu, b, dx, 1e-9, 20, metric=block)
    xb, _ = O.flex_solve(du, cu, b, dx, 1e-9, 20)
    peak = np.abs(xb).max()
    assert np.abs(xr - xb).max() < 1e-9 * peak
    x, rep = O.flex_solve(d, cr, b, dx, 1e-6, 200, metric=metric)
    assert rep["converged"], rep
    ax = O.flex_operator(d, cr, x, dx, metric)
    assert np.abs(ax - b).max() < 1e-3 * top


def test_the_operator_is_symmetric_and_the_preconditioner_is_spd():
    # The properties PCG needs (flexure.rs:1626-1629): <Au, v> = <u, Av> and <M^-1 u, v> symmetric.
    rng = np.random.default_rng(5)
    w, h, dx = 48, 24, 20_000.0
    te = patchy(w, h, 5.0, 60.0)
    d = np.vectorize(lambda t: O.rigidity_per_g(t, G))(te)
    c = np.full((h, w), RHO_M)
    u, v = rng.standard_normal((h, w)), rng.standard_normal((h, w))
    for precond in (O.PRECOND_REFERENCE, O.PRECOND_MEAN_D):
        mu, mv = O.flex_precondition(d, c, u, dx, precond), O.flex_precondition(d, c, v, dx, precond)
        a, b2 = float((mu * v).sum()), float((u * mv).sum())
        assert abs(a - b2) <= 1e-10 * max(abs(a), abs(b2))
        assert float((mu * u).sum()) > 0
    au, av = O.flex_operator(d, c, u, dx), O.flex_operator(d, c, v, dx)
    a, b2 = float((au * v).sum()), float((u * av).sum())
    assert abs(a - b2) <= 1e-12 * max(abs(a), abs(b2))


def test_the_relative_residual_rule_reaches_its_tolerance():
    # the benchmark's stopping rule (not the reference's): ||r|| / ||b|| <= tol, both preconditioners.
    w, h, dx = 64, 32, 10_000.0
    rng = np.random.default_rng(3)
    te = patchy(w, h, 8.0, 60.0)
    d = np.vectorize(lambda t: O.rigidity_per_g(t, G))(te)
    c = np.full((h, w), RHO_M)
    b = rng.standard_normal((h, w)) * 1e5
    for precond in (O.PRECOND_REFERENCE, O.PRECOND_MEAN_D):
        x, rep = O.flex_solve(d, c, b, dx, 1e-10, 2000, precond=precond, stop=O.STOP_REL_RESIDUAL)
        assert rep["converged"], rep
        true_rel = np.linalg.norm(b - O.flex_operator(d, c, x, dx)) / np.linalg.norm(b)
        assert true_rel < 1e-9, true_rel
