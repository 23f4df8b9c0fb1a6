"""Failure detection on the device, without faulting, trapping or hanging the GPU.

The reference turns a device timeout or a lost device into an error its caller handles
(deeptime-gpu/src/lib.rs:314-334; multigrid.rs:443-455). Here:

- A wait that runs out. Every wait of the TMA stencil on its tile barrier is bounded. With
  DT_STENCIL_WAIT_GIVE_UP=1 at dt_flex_create the waits give up without testing the barrier,
  the path a wait that ran out takes: the block waits (bounded) for its copies in flight to land,
  flags the fault and stops the solve, and the solve returns DT_DEVICE_ERROR. The context stays
  usable: another handle on the same device solves normally afterwards.
- Running out of memory. With DT_FAIL_ALLOC_AT=n the n-th device allocation of a create fails as
  cudaMalloc does when the device is full; the create returns DT_OOM and frees what it had
  allocated (the device's free memory is back where it was).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle as O  # noqa: E402
from deeptime_gpu import _lib as L  # noqa: E402
from deeptime_gpu import cube as C  # noqa: E402
from deeptime_gpu import diffusion as D  # noqa: E402
from deeptime_gpu import flexure as F  # noqa: E402
from deeptime_gpu import inputs as I  # noqa: E402
from tests.fixtures import cube_case  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED_RELIABLE])
def test_a_tile_wait_that_runs_out_is_a_device_error_and_the_context_survives(monkeypatch, precision):
    w, h, dx = 256, 128, 10_000.0  # rows of whole 64-cell tiles: the TMA stencil runs
    d, c, b = I.flexure_problem(w, h, 8.0, 77)
    monkeypatch.setenv("DT_STENCIL_WAIT_GIVE_UP", "1")
    bad = F.Solver(w, h, dx)
    monkeypatch.delenv("DT_STENCIL_WAIT_GIVE_UP")
    good = F.Solver(w, h, dx)
    p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=precision, tol=1e-8,
                 max_iterations=2000)
    with pytest.raises(L.DeepTimeError) as err:
        bad.solve_with(d, c, b, p)
    assert err.value.status == L.DT_DEVICE_ERROR and "ran out" in str(err.value)
    torch.cuda.synchronize()  # no sticky CUDA error
    x, rep = good.solve_with(d, c, b, p)
    assert rep.converged and rep.rel_residual <= 1e-8
    xo, _ = O.flex_solve(d, c, b, dx, 1e-12, 5000, precond=O.PRECOND_REFERENCE, stop=O.STOP_REL_RESIDUAL)
    assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
    with pytest.raises(L.DeepTimeError):  # the bad handle keeps giving up
        bad.solve_with(d, c, b, p)
    bad.close()
    good.close()


def _creates():
    n = 64
    slots = O.cube_topology(n)
    lap, areas, _, _ = cube_case(n, 9, slots)
    return {
        "flexure": lambda: F.Solver(2048, 1024, 2500.0),
        "diffusion": lambda: D.Workspace(D.Dims(2048, 1024, 2500.0, True)),
        "cube": lambda: C.CubeDiffusion(n, slots, lap, areas),
    }


@pytest.mark.parametrize("what", ["flexure", "diffusion", "cube"])
def test_an_allocation_that_fails_is_out_of_memory_and_leaks_nothing(monkeypatch, what):
    create = _creates()[what]
    torch.cuda.synchronize()
    ok = create()  # the first create may load code and size the context; measure after it
    ok.close()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    failed = 0
    for at in (1, 2, 5, 9, 14, 22):
        monkeypatch.setenv("DT_FAIL_ALLOC_AT", str(at))
        try:
            made = create()
        except L.DeepTimeError as e:
            assert e.status == L.DT_OOM and "DT_FAIL_ALLOC_AT" in str(e), e
            failed += 1
        else:
            made.close()  # fewer allocations than `at`: nothing failed
        monkeypatch.delenv("DT_FAIL_ALLOC_AT")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert failed >= 3
    # each failed create had up to 21 arrays of 16 MB; all of them were given back
    assert free0 - free1 < 16 << 20, (free0 - free1) / 2**20
    again = create()  # and the next create works
    again.close()
