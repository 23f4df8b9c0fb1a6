"""The cube grid's implicit diffusion on the device (dt_cube_*): the reference's
surface/cube/diffusion.rs::solve with DiffusionSolver::Multigrid, its multigrid V-cycle
(surface/cube/multigrid.rs). The grid's geometry is the caller's CubeGrid: the neighbour slots
(6 n^2 x 8, 0xFFFFFFFF where there is none), the coupling Laplacian's weights and the areas."""
import ctypes

import numpy as np

from . import _lib as L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class CubeDiffusion:
    def __init__(self, n: int, slots, lap, areas):
        self.n = int(n)
        self.cells = 6 * self.n * self.n
        slots = np.ascontiguousarray(slots, dtype=np.uint32).reshape(self.cells, 8)
        lap = _f64(lap).reshape(self.cells, 8)
        areas = _f64(areas).reshape(self.cells)
        handle = ctypes.c_void_p()
        L.check(L.lib().dt_cube_create(self.n, _ptr(slots), _ptr(lap), _ptr(areas), ctypes.byref(handle)))
        self._h = handle

    def close(self):
        if getattr(self, "_h", None):
            L.lib().dt_cube_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def levels(self) -> int:
        return L.lib().dt_cube_levels(self._h)

    def solve(self, h, kd, dt: float, tol_m: float):
        """One implicit step: returns (h', report); the report's error_m is the RMS residual."""
        h = _f64(h).copy()
        kd = _f64(kd)
        assert h.size == self.cells and kd.size == self.cells, "cells"
        rep = L.Report()
        st = L.lib().dt_cube_diff_solve(self._h, _ptr(h), _ptr(kd), float(dt), float(tol_m), ctypes.byref(rep))
        L.check(st, allow=(L.DT_OK, L.DT_NOT_CONVERGED))
        return h, rep

    def _map(self, fn, kd, dt, v):
        kd, v = _f64(kd), _f64(v)
        out = np.empty_like(v)
        L.check(getattr(L.lib(), fn)(self._h, _ptr(kd), float(dt), _ptr(v), _ptr(out)))
        return out

    def operator(self, kd, dt, x):
        return self._map("dt_cube_operator", kd, dt, x)

    def vcycle(self, kd, dt, r):
        return self._map("dt_cube_vcycle", kd, dt, r)

    def lod(self, kd, dt, h):
        return self._map("dt_cube_lod", kd, dt, h)
