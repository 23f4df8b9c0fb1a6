"""dt_flex_operator_dot_noalloc: the flexure operator and v.Av for callers that cannot allocate
device memory where they need them (a host code that gives the device to its own fixed arena, or
one that must not let cudaMalloc / cudaFree synchronise the device), against dt_flex_operator.

This file is collected last so that it also runs after every other test has used the device.
Tolerances: y is the same FP64 tile kernel as dt_flex_operator's, compared at 1e-13 relative;
v.Av is a deterministic sum in another order than numpy's, compared at 1e-12 relative.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from deeptime_gpu import _lib as L  # noqa: E402
from deeptime_gpu import flexure as F  # noqa: E402
from deeptime_gpu import inputs as I  # noqa: E402

pytestmark = pytest.mark.gpu


def call(lib, w, h, dx, d, c, v, y, vav, stream):
    return lib.dt_flex_operator_dot_noalloc(w, h, ctypes.c_double(dx), ctypes.c_void_p(d.data_ptr()),
                                            ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                            ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(vav.data_ptr()),
                                            ctypes.c_void_p(stream))


@pytest.mark.parametrize("w,h,dx", [(512, 256, 10_000.0), (1000, 37, 2_500.0)])
def test_two_calls_in_a_row_match_the_allocating_entry_point(w, h, dx):
    lib = L.lib()
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    want = []
    for seed in (3, 11):
        d, c, _ = I.flexure_problem(w, h, 8.0, seed)
        v = np.random.default_rng(seed).standard_normal((h, w)) * 50.0
        if w % 2 == 0 and h & (h - 1) == 0:
            y_ref = F.Solver(w, h, dx).operator(d, c, v)
        else:  # dt_flex_create takes power-of-two rasters only; the oracle stands in
            from oracle import oracle as O
            y_ref = O.flex_operator(d, c, v, dx)
        want.append((d, c, v, y_ref))
    for d, c, v, y_ref in want:
        td, tc, tv = (torch.from_numpy(a).to(dev) for a in (d, c, v))
        ty = torch.full((h, w), float("nan"), dtype=torch.float64, device=dev)
        tvav = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        assert call(lib, w, h, dx, td, tc, tv, ty, tvav, stream) == L.DT_OK, L.last_error()
        torch.cuda.synchronize()
        y = ty.cpu().numpy()
        assert np.linalg.norm(y - y_ref) <= 1e-13 * np.linalg.norm(y_ref)
        vav_ref = float(np.dot(v.ravel(), y_ref.ravel()))
        assert abs(tvav.item() - vav_ref) <= 1e-12 * abs(vav_ref)


def test_a_zero_vector_does_not_stick_and_oversize_rasters_are_refused():
    lib = L.lib()
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    w, h, dx = 256, 128, 10_000.0
    d, c, _ = I.flexure_problem(w, h, 8.0, 5)
    v = np.random.default_rng(5).standard_normal((h, w))
    td, tc, tv = (torch.from_numpy(a).to(dev) for a in (d, c, v))
    ty = torch.empty((h, w), dtype=torch.float64, device=dev)
    tvav = torch.empty((1,), dtype=torch.float64, device=dev)
    # v = 0 gives v.Av = 0, which the tile kernel's reduction flags as a breakdown; the next call
    # must start clean
    zero = torch.zeros_like(tv)
    assert call(lib, w, h, dx, td, tc, zero, ty, tvav, stream) == L.DT_OK, L.last_error()
    torch.cuda.synchronize()
    assert tvav.item() == 0.0 and torch.count_nonzero(ty).item() == 0
    assert call(lib, w, h, dx, td, tc, tv, ty, tvav, stream) == L.DT_OK, L.last_error()
    torch.cuda.synchronize()
    y_ref = F.Solver(w, h, dx).operator(d, c, v)
    assert np.linalg.norm(ty.cpu().numpy() - y_ref) <= 1e-13 * np.linalg.norm(y_ref)
    assert abs(tvav.item() - float(np.dot(v.ravel(), y_ref.ravel()))) <= 1e-12 * abs(tvav.item())
    # 16384 x 8208 needs 256 x 513 tiles, past the fixed scratch: refused before any device work
    assert call(lib, 16384, 8208, dx, td, tc, tv, ty, tvav, stream) == L.DT_UNSUPPORTED
    assert "fixed scratch" in L.last_error()
    # 64 x 1,100,000 fits the scratch (68,750 tiles) but not a launch's 65535 rows of tiles
    assert call(lib, 64, 1_100_000, dx, td, tc, tv, ty, tvav, stream) == L.DT_UNSUPPORTED
    assert "rows of tiles" in L.last_error()
