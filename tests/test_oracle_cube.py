"""The oracle's restatement of the cube grid's diffusion solve with its multigrid preconditioner
(surface/cube/diffusion.rs, surface/cube/multigrid.rs), pinned by the properties the reference's
own tests hold it to (surface/cube/tests.rs): the topology's neighbours are mutual, the operator
is symmetric, the V-cycle is a symmetric positive definite operator, the solve meets its RMS
tolerance and keeps the volume sum(a h) to round-off."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.fixtures import cube_case

NO = O.NO_CELL


@pytest.mark.parametrize("n", [2, 3, 8, 15])
def test_the_topology_is_mutual_and_misses_one_diagonal_at_each_cube_corner(n):
    s = O.cube_topology(n)
    cells = 6 * n * n
    assert s.shape == (cells, 8)
    for c in range(cells):
        for k in range(8):
            m = s[c, k]
            if m != NO:
                assert c in s[m], (c, k, m)
                assert m != c
        # a cell's eight neighbours are distinct
        have = [m for m in s[c] if m != NO]
        assert len(set(have)) == len(have)
    # only diagonals go missing, one at each of a face's four corner cells
    assert (s[:, 0::2] != NO).all()
    assert int((s == NO).sum()) == 6 * 4


@pytest.mark.parametrize("n", [1, 2, 3, 8, 15, 64])
def test_the_packages_topology_is_the_oracles(n):
    # the slots a caller builds with the package (deeptime_gpu.cube.topology) are the oracle's
    from deeptime_gpu import cube as C

    assert np.array_equal(C.topology(n), O.cube_topology(n))


def test_the_operator_is_symmetric():
    n = 8
    s = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, 1, s)
    rng = np.random.default_rng(2)
    u, v = rng.standard_normal(6 * n * n), rng.standard_normal(6 * n * n)
    au = O.cube_operator(n, s, lap, areas, kd, 3.0, u)
    av = O.cube_operator(n, s, lap, areas, kd, 3.0, v)
    assert abs(u @ av - v @ au) <= 1e-12 * abs(u @ av)
    # rows sum to mu: A 1 = mu
    one = O.cube_operator(n, s, lap, areas, kd, 3.0, np.ones(6 * n * n))
    mean = areas.sum() / areas.size
    assert np.allclose(one, areas / mean, rtol=1e-12)


def test_the_cycle_is_symmetric_positive_definite():
    n = 16
    s = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, 3, s)
    rng = np.random.default_rng(4)
    r1, r2 = rng.standard_normal(6 * n * n), rng.standard_normal(6 * n * n)
    z1 = O.cube_vcycle(n, s, lap, areas, kd, 5.0, r1)
    z2 = O.cube_vcycle(n, s, lap, areas, kd, 5.0, r2)
    assert abs(r1 @ z2 - r2 @ z1) <= 1e-5 * max(abs(r1 @ z2), 1e-30)
    assert r1 @ z1 > 0 and r2 @ z2 > 0


@pytest.mark.parametrize("n,dt", [(8, 2.0), (16, 50.0), (13, 10.0)])
def test_the_solve_meets_its_tolerance_and_keeps_the_volume(n, dt):
    s = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, n, s)
    tol = 1e-6
    x, its = O.cube_diff_solve(n, s, lap, areas, kd, dt, tol, h)
    assert 0 < its < 400
    mean = areas.sum() / areas.size
    mu = areas / mean
    ax = O.cube_operator(n, s, lap, areas, kd, dt, x)
    # the put-back moves x by the residual's sum, so the RMS residual is checked on its mean-free part
    r = mu * h - ax
    assert np.sqrt(np.mean((r - r.mean()) ** 2)) < 10 * tol
    assert abs((mu * x).sum() - (mu * h).sum()) <= 1e-9 * np.abs(mu * h).sum()


def test_the_first_guess_is_a_smoothing_of_the_field():
    n = 12
    s = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, 7, s)
    x = O.cube_lod(n, s, lap, areas, kd, 4.0, h)
    assert np.isfinite(x).all()
    assert np.std(x) < np.std(h)
    # no coupling: the first guess is the field itself
    x0 = O.cube_lod(n, s, lap, areas, np.zeros_like(kd), 4.0, h)
    assert np.array_equal(x0, h)


def test_a_level_field_stays_level():
    # A constant h is its own implicit step: A h = mu h, so the LOD guess returns it and CG stops at once
    n = 10
    s = O.cube_topology(n)
    lap, areas, kd, _ = cube_case(n, 11, s)
    h = np.full(6 * n * n, 123.25)
    x, its = O.cube_diff_solve(n, s, lap, areas, kd, 30.0, 1e-6, h)
    assert its == 0
    assert np.allclose(x, h, rtol=1e-12, atol=0)
