"""The cube grid's diffusion solve on the device (dt_cube_*) against the oracle's restatement of
the reference (surface/cube/diffusion.rs, surface/cube/multigrid.rs), through the C ABI.

Tolerances: the operator and the LOD first guess are FP64 with the reference's operation order,
compared at 1e-14 relative; the V-cycle is FP32, compared at 1e-6 relative; solves stop at an RMS
residual of tol, so the two answers are compared at 100 tol (m) absolute, their iteration counts
within one, and the volume sum(mu h) to 1e-9 relative."""
import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import cube as C
from tests.fixtures import cube_case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module", params=[8, 13, 32])
def case(request):
    n = request.param
    slots = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, n + 100, slots)
    return n, slots, lap, areas, kd, h, C.CubeDiffusion(n, slots, lap, areas)


def test_operator_matches_the_oracle(case):
    n, slots, lap, areas, kd, h, dev = case
    x = np.random.default_rng(1).standard_normal(6 * n * n)
    assert rel(dev.operator(kd, 7.0, x), O.cube_operator(n, slots, lap, areas, kd, 7.0, x)) < 1e-14


def test_lod_first_guess_matches_the_oracle(case):
    n, slots, lap, areas, kd, h, dev = case
    assert rel(dev.lod(kd, 7.0, h), O.cube_lod(n, slots, lap, areas, kd, 7.0, h)) < 1e-14


@pytest.mark.parametrize("n", [33, 70, 256])
def test_the_chunked_line_solves_match_the_serial_walks_and_the_oracle(n, monkeypatch):
    # lines of n cells in chunks of 32 (two with a last chunk of one cell, three with a ragged
    # last, eight) against one serial walk a line (DT_CUBE_LOD_CHUNKED=0 at create) and the oracle
    slots = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, n + 100, slots)
    chunked = C.CubeDiffusion(n, slots, lap, areas)
    monkeypatch.setenv("DT_CUBE_LOD_CHUNKED", "0")
    serial = C.CubeDiffusion(n, slots, lap, areas)
    monkeypatch.delenv("DT_CUBE_LOD_CHUNKED")
    want = O.cube_lod(n, slots, lap, areas, kd, 7.0, h)
    got, walk = chunked.lod(kd, 7.0, h), serial.lod(kd, 7.0, h)
    assert rel(walk, want) < 1e-14
    assert rel(got, want) < 1e-14 and rel(got, walk) < 1e-14, (rel(got, want), rel(got, walk))
    chunked.close()
    serial.close()


def test_vcycle_matches_the_oracle(case):
    n, slots, lap, areas, kd, h, dev = case
    r = np.random.default_rng(2).standard_normal(6 * n * n)
    assert rel(dev.vcycle(kd, 7.0, r), O.cube_vcycle(n, slots, lap, areas, kd, 7.0, r)) < 1e-6


@pytest.mark.parametrize("dt", [0.5, 7.0, 60.0])
def test_solve_matches_the_oracle_and_keeps_the_volume(case, dt):
    n, slots, lap, areas, kd, h, dev = case
    tol = 1e-6
    want, its = O.cube_diff_solve(n, slots, lap, areas, kd, dt, tol, h)
    got, rep = dev.solve(h, kd, dt, tol)
    assert rep.converged and rep.error_m <= tol
    assert abs(rep.iterations - its) <= 1, (rep.iterations, its)
    assert np.abs(got - want).max() < 100 * tol
    mu = areas / (areas.sum() / areas.size)
    assert abs((mu * got).sum() - (mu * h).sum()) <= 1e-9 * np.abs(mu * h).sum()


def test_no_step_leaves_the_field_as_it_was(case):
    n, slots, lap, areas, kd, h, dev = case
    for dt in (0.0, float("nan")):
        got, rep = dev.solve(h, kd, dt, 1e-6)
        assert rep.iterations == 0 and np.array_equal(got, h)


def test_the_hierarchy_reaches_64_cells():
    n = 32
    slots = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, 1, slots)
    dev = C.CubeDiffusion(n, slots, lap, areas)
    # sides 32, 16, 8, 4, 2: the last level 24 cells (the first at or below 64)
    assert dev.levels == 5


def test_a_level_field_stays_level_on_the_device(case):
    n, slots, lap, areas, kd, h, dev = case
    level = np.full(6 * n * n, -42.5)
    got, rep = dev.solve(level, kd, 30.0, 1e-6)
    assert rep.iterations == 0
    assert np.allclose(got, level, rtol=1e-12, atol=0)


@pytest.mark.parametrize("n", [8, 32, 64])
def test_the_one_block_coarse_cycle_is_bit_for_bit_the_separate_launches(n, monkeypatch):
    """The coarse levels' cycle in one block (the default) against every level launching its own
    kernels (DT_CUBE_FUSE_CELLS=0 at dt_cube_create): the same phases in the same order, so the
    same bits. At n = 8 every level runs in the block; at 32 and 64 the finer levels launch."""
    slots = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, n + 200, slots)
    r = np.random.default_rng(n).standard_normal(6 * n * n)
    fused = C.CubeDiffusion(n, slots, lap, areas)
    monkeypatch.setenv("DT_CUBE_FUSE_CELLS", "0")
    apart = C.CubeDiffusion(n, slots, lap, areas)
    monkeypatch.delenv("DT_CUBE_FUSE_CELLS")
    for dt in (7.0, 60.0):
        a, b = fused.vcycle(kd, dt, r), apart.vcycle(kd, dt, r)
        assert np.array_equal(a, b), float(np.abs(a - b).max())
        # twice in a row: the second cycle runs on the other buffer layout
        assert np.array_equal(fused.vcycle(kd, dt, r), apart.vcycle(kd, dt, r))
    xa, ra = fused.solve(h, kd, 7.0, 1e-6)
    xb, rb = apart.solve(h, kd, 7.0, 1e-6)
    assert ra.iterations == rb.iterations and np.array_equal(xa, xb)


@pytest.mark.parametrize("n", [13, 64])
def test_the_device_loop_is_bit_for_bit_the_host_driven_one(n, monkeypatch):
    """The CG loop as a CUDA graph (the default: a WHILE node, the iteration's tail under an IF
    node) against the loop driven from the host (DT_CUBE_HOST_LOOP=1 at create): the same kernels
    in the same order, so the same iterations and the same bits, twice in a row on each handle."""
    slots = O.cube_topology(n)
    lap, areas, kd, h = cube_case(n, n + 300, slots)
    graph = C.CubeDiffusion(n, slots, lap, areas)
    monkeypatch.setenv("DT_CUBE_HOST_LOOP", "1")
    host = C.CubeDiffusion(n, slots, lap, areas)
    monkeypatch.delenv("DT_CUBE_HOST_LOOP")
    for dt in (7.0, 60.0, 7.0):
        xg, rg = graph.solve(h, kd, dt, 1e-6)
        xh, rh = host.solve(h, kd, dt, 1e-6)
        assert rg.iterations == rh.iterations and rg.converged == rh.converged
        assert np.array_equal(xg, xh), float(np.abs(xg - xh).max())
