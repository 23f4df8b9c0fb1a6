"""The flexure step's grid helpers on device rasters (dt_grid_*_dev): restrict_by, prolong_const,
prolong_linear and binomial (flexure.rs:1745-1844) and box_blur (grid.rs:224-270), bit-for-bit
with the reference. Rasters are CUDA float64 tensors of shape (h, w), row-major; each call runs on
torch's current stream."""
import ctypes

from . import _lib as L


def _torch():
    import torch

    return torch


def _check(t):
    torch = _torch()
    assert t.is_cuda and t.dtype == torch.float64 and t.dim() == 2 and t.is_contiguous(), "a contiguous (h, w) CUDA float64 raster"


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def restrict(fine, f: int):
    """The mean of each f x f block (restrict_by): (h // f, w // f)."""
    _check(fine)
    h, w = fine.shape
    out = _torch().empty((h // f, w // f), dtype=fine.dtype, device=fine.device)
    L.check(L.lib().dt_grid_restrict_dev(w, h, f, _p(fine), _p(out), _stream()))
    return out


def prolong_const(coarse, f: int):
    """Each coarse value on its f x f cells: (hs f, ws f)."""
    _check(coarse)
    hs, ws = coarse.shape
    out = _torch().empty((hs * f, ws * f), dtype=coarse.dtype, device=coarse.device)
    L.check(L.lib().dt_grid_prolong_const_dev(ws, hs, f, _p(coarse), _p(out), _stream()))
    return out


def prolong_linear(coarse, f: int):
    """Bilinear from the coarse cells' centres, x wrapping, rows clamped: (hs f, ws f)."""
    _check(coarse)
    hs, ws = coarse.shape
    out = _torch().empty((hs * f, ws * f), dtype=coarse.dtype, device=coarse.device)
    L.check(L.lib().dt_grid_prolong_linear_dev(ws, hs, f, _p(coarse), _p(out), _stream()))
    return out


def binomial(v, passes: int):
    """`passes` of [1/4, 1/2, 1/4] along x (wrapping) then y (rows clamped), in place."""
    _check(v)
    h, w = v.shape
    scratch = _torch().empty_like(v)
    L.check(L.lib().dt_grid_binomial_dev(w, h, passes, _p(v), _p(scratch), _stream()))
    return v


def box_blur(v, r: int, passes: int, wrap_x: bool = True):
    """`passes` of the radius-r running box along x (wrapping or clamped) then y (reflected), in place."""
    _check(v)
    h, w = v.shape
    scratch = _torch().empty_like(v)
    L.check(L.lib().dt_grid_box_blur_dev(w, h, int(wrap_x), r, passes, _p(v), _p(scratch), _stream()))
    return v
