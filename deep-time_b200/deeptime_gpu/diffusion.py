"""The implicit diffusion solve behind the reference's interface, on the B200.

`solve(ws, d, h, kd, dt, solver, tol_m)` mirrors `diffusion::solve`
(crates/deeptime-core/src/surface/diffusion.rs:77-97): `h` is the right-hand side on entry and the
solution on return, `kd` the diffusivity per cell (m^2/yr), `dt` the step (yr); it returns the
iterations. `Workspace` holds the device handle for one raster shape (the reference's `Workspace`
keeps the solve's vectors, diffusion.rs:214-260), `Dims` the raster (grid.rs:11-17). Only the
multigrid solver is on the device (`DiffusionSolver::Multigrid`, the surface stage's default);
`solve_with` exposes the benchmark's variants (red-black cycle, FP64 cycle, mixed precision,
relative-residual rule). Every call goes through the C ABI; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .flexure import SolveReport, _f64, _ptr

MULTIGRID = "multigrid"


@dataclass(frozen=True)
class Dims:
    w: int
    h: int
    dx: float
    wrap_x: bool

    def cells(self):
        return self.w * self.h


class DiffParams(ctypes.Structure):
    _fields_ = [("cycle", ctypes.c_int), ("precision", ctypes.c_int), ("stop", ctypes.c_int), ("tol", ctypes.c_double),
                ("max_iterations", ctypes.c_int), ("first_guess", ctypes.c_int), ("inner_tol", ctypes.c_double),
                ("max_refinements", ctypes.c_int), ("host_loop", ctypes.c_int)]


def _declare(lib):
    if getattr(lib, "_diff_declared", False):
        return
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.dt_diff_default_params.argtypes = [ctypes.POINTER(DiffParams)]
    lib.dt_diff_create.argtypes = [i, i, d, i, ctypes.POINTER(vp)]
    lib.dt_diff_destroy.argtypes = [vp]
    lib.dt_diff_set_stream.argtypes = [vp, vp]
    for name in ("dt_diff_solve", "dt_diff_solve_dev"):
        getattr(lib, name).argtypes = [vp, vp, vp, d, ctypes.POINTER(DiffParams), ctypes.POINTER(L.Report)]
    lib.dt_diff_operator.argtypes = [vp, vp, d, vp, vp]
    lib.dt_diff_vcycle.argtypes = [vp, vp, d, i, vp, vp, ctypes.POINTER(i)]
    lib.dt_diff_lod.argtypes = [vp, vp, vp, d, vp]
    lib.dt_diff_profile_kernels.argtypes = [vp, vp, d, i, vp, vp]
    lib._diff_declared = True


def params(cycle=L.CYCLE_JACOBI, precision=L.DIFF_FP64_CG_FP32_CYCLE, stop=L.STOP_RMS_RESIDUAL, tol=1e-5,
           max_iterations=400, first_guess=True, inner_tol=1e-5, max_refinements=8, host_loop=0) -> DiffParams:
    lib = L.lib()
    _declare(lib)
    p = DiffParams()
    lib.dt_diff_default_params(ctypes.byref(p))
    p.cycle, p.precision, p.stop, p.tol = cycle, precision, stop, tol
    p.max_iterations, p.first_guess, p.inner_tol = max_iterations, int(bool(first_guess)), inner_tol
    p.max_refinements, p.host_loop = max_refinements, host_loop
    return p


class Workspace:
    """The device state of one raster shape (handle, buffers, multigrid levels, graphs)."""

    def __init__(self, dims: Dims):
        lib = L.lib()
        _declare(lib)
        self.dims = dims
        handle = ctypes.c_void_p()
        L.check(lib.dt_diff_create(dims.w, dims.h, float(dims.dx), int(dims.wrap_x), ctypes.byref(handle)))
        self._h = handle

    def close(self):
        if getattr(self, "_h", None):
            L.lib().dt_diff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve_with(self, h, kd, dt, p: DiffParams):
        h, kd = _f64(h).copy(), _f64(kd)
        assert h.size == self.dims.cells() and kd.size == self.dims.cells(), "raster size"
        rep = L.Report()
        st = L.lib().dt_diff_solve(self._h, _ptr(h), _ptr(kd), float(dt), ctypes.byref(p), ctypes.byref(rep))
        L.check(st, allow=(L.DT_OK, L.DT_NOT_CONVERGED))
        return h, SolveReport(rep.iterations, rep.error_m, bool(rep.converged), rep.rel_residual, rep.refinements, False,
                              float("nan"), rep.device_ms, rep.kernel_launches, st)

    def operator(self, kd, dt, x):
        kd, x = _f64(kd), _f64(x)
        y = np.empty_like(x)
        L.check(L.lib().dt_diff_operator(self._h, _ptr(kd), float(dt), _ptr(x), _ptr(y)))
        return y

    def lod(self, h, kd, dt):
        """The LOD splitting's first guess from h (diffusion.rs:370-489), as the solve starts from."""
        h, kd = _f64(h), _f64(kd)
        x = np.empty_like(h)
        L.check(L.lib().dt_diff_lod(self._h, _ptr(h), _ptr(kd), float(dt), _ptr(x)))
        return x

    def vcycle(self, kd, dt, r, cycle=L.CYCLE_JACOBI):
        kd, r = _f64(kd), _f64(r)
        z = np.empty(r.shape, dtype=np.float32)
        levels = ctypes.c_int(0)
        L.check(L.lib().dt_diff_vcycle(self._h, _ptr(kd), float(dt), cycle, _ptr(r), ctypes.c_void_p(z.ctypes.data),
                                       ctypes.byref(levels)))
        return z, levels.value

    # the kernels dt_diff_profile_kernels times, in its order
    PROFILE_KERNELS = ("apply_fp64", "apply_fp32", "rb2_pre_fp32", "rb2_post_fp32", "rb2_pre_fp64", "rb2_post_fp64")

    def profile_kernels(self, kd, dt, reps=20):
        """{name: (ms a launch, algorithmic bytes a launch)} of the finest level's hot kernels for
        the operator of kd and dt, each launch timed alone after an L2 flush."""
        kd = _f64(kd)
        k = len(self.PROFILE_KERNELS)
        ms, by = (ctypes.c_double * k)(), (ctypes.c_double * k)()
        L.check(L.lib().dt_diff_profile_kernels(self._h, _ptr(kd), float(dt), int(reps), ms, by))
        return {name: (ms[q], by[q]) for q, name in enumerate(self.PROFILE_KERNELS)}


def solve(ws: Workspace, d: Dims, h: np.ndarray, kd, dt: float, solver: str = MULTIGRID, tol_m: float = 1e-5) -> int:
    """diffusion::solve with DiffusionSolver::Multigrid: `h` (a float64 array of d.cells() values)
    becomes the solution in place; returns the conjugate-gradient iterations."""
    if solver != MULTIGRID:
        raise L.DeepTimeError(L.DT_UNSUPPORTED, "only the multigrid solver has a device path")
    assert ws.dims == d, "workspace raster"
    assert h.dtype == np.float64 and h.flags.c_contiguous, "h must be a contiguous float64 array"
    x, rep = ws.solve_with(h, kd, dt, params(tol=tol_m))
    h[...] = x.reshape(h.shape)
    return rep.iterations
