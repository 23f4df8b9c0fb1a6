"""The cube grid's implicit diffusion on the device (dt_cube_*): the reference's
surface/cube/diffusion.rs::solve with DiffusionSolver::Multigrid, its multigrid V-cycle
(surface/cube/multigrid.rs). The grid's geometry is the caller's CubeGrid: the neighbour slots
(6 n^2 x 8, 0xFFFFFFFF where there is none), the coupling Laplacian's weights and the areas."""
import ctypes

import numpy as np

from . import _lib as L


NO_CELL = 0xFFFFFFFF

# The cube's face adjacency (deeptime-format/src/cube.rs:321-369): for face F0, F1, F2, F3, N, S
# and side east, south, west, north, the face across the side, the clockwise quarter turns that
# take a cell's frame onto that face's, and the face's shift in cells of n (x, then y).
_ACROSS = np.array([
    [[1, 0, -1, 0], [5, 0, 0, -1], [3, 0, 1, 0], [4, 0, 0, 1]],
    [[2, 0, -1, 0], [5, 1, 2, 0], [0, 0, 1, 0], [4, 3, 1, 1]],
    [[3, 0, -1, 0], [5, 2, 1, 2], [1, 0, 1, 0], [4, 2, 1, 0]],
    [[0, 0, -1, 0], [5, 3, -1, 1], [2, 0, 1, 0], [4, 1, 0, 0]],
    [[1, 1, 1, -1], [0, 0, 0, -1], [3, 3, 0, 0], [2, 2, 1, 0]],
    [[1, 3, 0, 2], [2, 2, 1, 2], [3, 1, 1, 1], [0, 0, 0, 1]],
], dtype=np.int64)
# the eight neighbour slots' offsets E, NE, N, NW, W, SW, S, SE, j growing southward
# (surface/grid.rs:21-30)
_OFFSETS = np.array([[1, 0], [1, -1], [0, -1], [-1, -1], [-1, 0], [-1, 1], [0, 1], [1, 1]], dtype=np.int64)


def topology(n: int) -> np.ndarray:
    """The 6 n^2 cells' eight neighbour slots (sphere/cube.rs:76-93), (6 n^2, 8) uint32: cell
    (face f, column i, row j) is f n^2 + j n + i; a step off a face lands on the face across that
    side, in its frame; a step off a corner (both coordinates outside) has no cell (NO_CELL)."""
    n = int(n)
    c = np.arange(6 * n * n, dtype=np.int64)
    face, rem = c // (n * n), c % (n * n)
    i = (rem % n)[:, None] + _OFFSETS[:, 0]
    j = (rem // n)[:, None] + _OFFSETS[:, 1]
    out_i, out_j = (i < 0) | (i >= n), (j < 0) | (j >= n)
    side = np.where(i >= n, 0, np.where(i < 0, 2, np.where(j >= n, 1, 3)))
    a = _ACROSS[np.broadcast_to(face[:, None], i.shape), side]
    turns = a[..., 1]
    rx = np.select([turns == 1, turns == 2, turns == 3], [-j - 1, -i - 1, j], i)
    rz = np.select([turns == 1, turns == 2, turns == 3], [i, -j - 1, -i - 1], j)
    inside = ~out_i & ~out_j
    f2 = np.where(inside, face[:, None], a[..., 0])
    i2 = np.where(inside, i, rx + n * a[..., 2])
    j2 = np.where(inside, j, rz + n * a[..., 3])
    far = (i < -n) | (i >= 2 * n) | (j < -n) | (j >= 2 * n)
    return np.where((out_i & out_j) | far, NO_CELL, f2 * n * n + j2 * n + i2).astype(np.uint32)


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
