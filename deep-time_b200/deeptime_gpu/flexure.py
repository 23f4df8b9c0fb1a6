"""The flexure solver behind the reference's interface, on the B200.

`Solver` mirrors `flexure::Solver` (crates/deeptime-core/src/surface/flexure.rs:1471-1741):
`Solver(w, h, dx)` / `Solver.with_metric(w, h, dx, metric)` (:1524-1530), `solve(d, c, b,
tolerance_m, max_iterations) -> (x, SolveReport)` (:1680-1687) with the reference's stopping rule
(max |z| < tolerance_m) and preconditioner (the 3-level ln(alpha) bank inside damped Jacobi
sweeps), `operator` (:1606) and `bend` (:1598). Like the reference it panics (here: raises
AssertionError) on a size mismatch. `solve_with` exposes the other stopping rule, the mean-D
preconditioner, mixed precision and warm starts.

Every call goes through the C ABI of libdeeptime_gpu.so; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class SolveReport:
    """flexure.rs:947-952, plus this backend's extra facts."""
    iterations: int
    error_m: float
    converged: bool
    rel_residual: float = float("nan")
    refinements: int = 0
    warm_start_accepted: bool = False
    warm_start_rel_residual: float = float("nan")
    device_ms: float = float("nan")
    kernel_launches: int = 0
    status: int = 0


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def row_metric_from_sin_faces(sin_faces, f: int = 1):
    """RowMetric::from_sin_faces (flexure.rs:977-1000): the sphere's row metric of a raster whose
    row boundaries sit at the sines of latitude `sin_faces` (h f + 1 of them, every f-th taken).
    a_j = 1 / max(1 - m_j^2, least) with m_j the mean of row j's two faces and least half the
    largest step between faces (at least 1e-12); b_k = 1 - s_k^2 inside, 0 at the raster's edges.
    Returns (a, b) for Solver(w, h, dx, (a, b))."""
    f = max(int(f), 1)
    s = np.clip(_f64(sin_faces)[::f], -1.0, 1.0)
    h = (len(sin_faces) - 1) // f
    s = s[: h + 1]
    full = float(np.max(np.abs(np.diff(s)))) if h > 0 else 0.0
    least = max(0.5 * full, 1e-12)
    m = 0.5 * (s[:-1] + s[1:])
    a = 1.0 / np.maximum(1.0 - m * m, least)
    b = 1.0 - s * s
    b[0] = b[-1] = 0.0
    return a, b


def params(precond=L.PRECOND_REFERENCE, stop=L.STOP_MAX_Z, precision=L.PREC_FP64, warm_start=L.WARM_NONE, tol=2.0,
           max_iterations=60, inner_tol=1e-5, max_refinements=8, host_loop=0) -> L.FlexParams:
    p = L.FlexParams()
    L.lib().dt_flex_default_params(ctypes.byref(p))
    p.precond, p.stop, p.precision, p.warm_start = precond, stop, precision, warm_start
    p.tol, p.max_iterations, p.inner_tol, p.max_refinements = tol, max_iterations, inner_tol, max_refinements
    p.host_loop = host_loop
    return p


class Solver:
    def __init__(self, w: int, h: int, dx: float, metric=None):
        self.w, self.h, self.dx = int(w), int(h), float(dx)
        handle = ctypes.c_void_p()
        ma = mb = None
        if metric is not None:
            a, b = _f64(metric[0]), _f64(metric[1])
            if len(a) == h and len(b) == h + 1:  # flexure.rs:1531 keeps a metric of the right size only
                ma, mb = _ptr(a), _ptr(b)
        L.check(L.lib().dt_flex_create(self.w, self.h, self.dx, ma, mb, ctypes.byref(handle)))
        self._h = handle

    @classmethod
    def with_metric(cls, w, h, dx, metric):
        return cls(w, h, dx, metric)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().dt_flex_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_sizes(self, *arrays):
        n = self.w * self.h
        assert all(a.size == n for a in arrays), "raster size"

    def solve(self, d, c, b, tolerance_m: float, max_iterations: int):
        """The reference's Solver::solve: PCG from x = 0 until max |z| < tolerance_m (metres)."""
        return self.solve_with(d, c, b, params(tol=tolerance_m, max_iterations=max_iterations))

    def solve_with(self, d, c, b, p: L.FlexParams, x0=None):
        d, c, b = _f64(d), _f64(c), _f64(b)
        self._check_sizes(d, c, b)
        x = np.zeros_like(b) if x0 is None else _f64(x0).copy()
        rep = L.Report()
        st = L.lib().dt_flex_solve(self._h, _ptr(d), _ptr(c), _ptr(b), _ptr(x), ctypes.byref(p), ctypes.byref(rep))
        L.check(st, allow=(L.DT_OK, L.DT_NOT_CONVERGED))
        return x.reshape(b.shape), SolveReport(rep.iterations, rep.error_m, bool(rep.converged), rep.rel_residual,
                                               rep.refinements, bool(rep.warm_start_accepted),
                                               rep.warm_start_rel_residual, rep.device_ms, rep.kernel_launches, st)

    def operator(self, d, c, v):
        d, c, v = _f64(d), _f64(c), _f64(v)
        self._check_sizes(d, c, v)
        y = np.empty_like(v)
        L.check(L.lib().dt_flex_operator(self._h, _ptr(d), _ptr(c), _ptr(v), _ptr(y)))
        return y

    def bend(self, d, v):
        d, v = _f64(d), _f64(v)
        self._check_sizes(d, v)
        y = np.empty_like(v)
        L.check(L.lib().dt_flex_bend(self._h, _ptr(d), _ptr(v), _ptr(y)))
        return y

    def precondition(self, d, c, r, precond=L.PRECOND_REFERENCE, precision=L.PREC_FP64):
        d, c, r = _f64(d), _f64(c), _f64(r)
        self._check_sizes(d, c, r)
        z = np.empty_like(r)
        L.check(L.lib().dt_flex_precondition(self._h, _ptr(d), _ptr(c), _ptr(r), _ptr(z), precond, precision))
        return z
