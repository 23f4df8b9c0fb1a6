"""Test infrastructure only: numpy-facing ctypes bindings of the CPU oracle (liboracle.so).

The oracle restates the reference's CPU solvers (crates/deeptime-core/src/surface/flexure.rs,
surface/diffusion.rs, surface/diffusion/multigrid.rs); each C function cites the reference lines it
follows. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

PRECOND_REFERENCE, PRECOND_MEAN_D = 0, 1
STOP_MAX_Z, STOP_REL_RESIDUAL, STOP_RMS_RESIDUAL = 0, 1, 2
CYCLE_JACOBI, CYCLE_RBGS = 0, 1

RHO_MANTLE = 3300.0
RHO_WATER = 1030.0


class Report(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("error_m", ctypes.c_double),
        ("rel_residual", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build() -> str:
    """Compile liboracle.so with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        L.dto_rigidity_per_g.restype = d
        L.dto_rigidity_per_g.argtypes = [d, d]
        L.dto_flexural_parameter_m.restype = d
        L.dto_flexural_parameter_m.argtypes = [d]
        L.dto_diff_vcycle.restype = d
        L.dto_submarine_kd.restype = d
        L.dto_submarine_kd.argtypes = [d, d, d, d, d]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


D = ctypes.c_double


def set_threads(n: int) -> int:
    """Run the oracle's OpenMP loops on n threads (n <= 0: all host threads); returns the count."""
    lib().dto_set_threads(int(n))
    return int(lib().dto_threads())


def rigidity_per_g(te_km: float, g: float) -> float:
    return lib().dto_rigidity_per_g(te_km, g)


def flexural_parameter_m(d_per_g: float) -> float:
    return lib().dto_flexural_parameter_m(d_per_g)


def spectral_roundtrip(v: np.ndarray, dx: float) -> np.ndarray:
    h, w = v.shape
    v = _f64(v)
    out = np.empty_like(v)
    lib().dto_flex_spectral_roundtrip(w, h, D(dx), _p(v), _p(out))
    return out


def flex_operator(d, c, v, dx, metric=None):
    h, w = v.shape
    d, c, v = _f64(d), _f64(c), _f64(v)
    ma, mb = (None, None) if metric is None else (_f64(metric[0]), _f64(metric[1]))
    y = np.empty_like(v)
    lib().dto_flex_operator(w, h, D(dx), _p(ma), _p(mb), _p(d), _p(c), _p(v), _p(y))
    return y


def flex_bend(d, v, dx):
    h, w = v.shape
    d, v = _f64(d), _f64(v)
    y = np.empty_like(v)
    lib().dto_flex_bend(w, h, D(dx), _p(d), _p(v), _p(y))
    return y


def flex_precondition(d, c, r, dx, precond=PRECOND_REFERENCE, metric=None):
    h, w = r.shape
    d, c, r = _f64(d), _f64(c), _f64(r)
    ma, mb = (None, None) if metric is None else (_f64(metric[0]), _f64(metric[1]))
    z = np.empty_like(r)
    lib().dto_flex_precondition(w, h, D(dx), _p(ma), _p(mb), _p(d), _p(c), _p(r), _p(z), precond)
    return z


def flex_bank(d, c, dx):
    h, w = d.shape
    d, c = _f64(d), _f64(c)
    node_d = np.zeros(3)
    c_ref = ctypes.c_double(0)
    weights = np.zeros((3, h, w))
    k = lib().dto_flex_bank(w, h, D(dx), _p(d), _p(c), _p(node_d), ctypes.byref(c_ref), _p(weights))
    return node_d[:k].copy(), c_ref.value, (weights[:k].copy() if k > 1 else None)


def flex_solve(d, c, b, dx, tol, max_it, precond=PRECOND_REFERENCE, stop=STOP_MAX_Z, metric=None):
    """The reference's Solver::solve (PCG from x = 0); returns (x, report dict)."""
    h, w = b.shape
    d, c, b = _f64(d), _f64(c), _f64(b)
    ma, mb = (None, None) if metric is None else (_f64(metric[0]), _f64(metric[1]))
    x = np.zeros_like(b)
    rep = Report()
    lib().dto_flex_solve(w, h, D(dx), _p(ma), _p(mb), _p(d), _p(c), _p(b), _p(x), D(tol), int(max_it), precond, stop,
                         ctypes.byref(rep))
    return x, rep.as_dict()


def row_metric_from_sin_faces(sin_faces, f=1):
    sin_faces = _f64(sin_faces)
    h = (len(sin_faces) - 1) // max(f, 1)
    a, b = np.zeros(h), np.zeros(h + 1)
    lib().dto_row_metric_from_sin_faces(_p(sin_faces), len(sin_faces), f, _p(a), _p(b))
    return a, b


def box_blur(v, r, passes, wrap=True):
    v = _f64(v).copy()
    h, w = v.shape
    lib().dto_box_blur(w, h, int(wrap), _p(v), r, passes)
    return v


def restrict_by(v, f):
    """flexure.rs:1773-1795: the mean of each f x f block."""
    v = _f64(v)
    h, w = v.shape
    out = np.empty((h // f, w // f))
    lib().dto_restrict_by(w, h, f, _p(v), _p(out))
    return out


def prolong_const(v, f):
    """flexure.rs:1803-1813."""
    v = _f64(v)
    hs, ws = v.shape
    out = np.empty((hs * f, ws * f))
    lib().dto_prolong_const(ws, hs, f, _p(v), _p(out))
    return out


def prolong_linear(v, f):
    """flexure.rs:1816-1844: bilinear from the coarse cells' centres, x wrapping, rows clamped."""
    v = _f64(v)
    hs, ws = v.shape
    out = np.empty((hs * f, ws * f))
    lib().dto_prolong_linear(ws, hs, f, _p(v), _p(out))
    return out


def binomial(v, passes):
    """flexure.rs:1745-1762: [1/4, 1/2, 1/4] along x (wrapping), then y (rows clamped)."""
    v = _f64(v).copy()
    h, w = v.shape
    lib().dto_binomial(w, h, passes, _p(v))
    return v


NO_CELL = 0xFFFFFFFF


def cube_topology(n):
    """sphere/cube.rs:76-93: the 6 n^2 cells' eight neighbour slots (E, NE, N, NW, W, SW, S, SE)."""
    slots = np.zeros((6 * n * n, 8), dtype=np.uint32)
    lib().dto_cube_topology(n, _p(slots))
    return slots


def _cube_args(n, slots, lap, areas, kd):
    return (np.ascontiguousarray(slots, dtype=np.uint32), _f64(lap), _f64(areas), _f64(kd))


def cube_operator(n, slots, lap, areas, kd, dt, x):
    slots, lap, areas, kd = _cube_args(n, slots, lap, areas, kd)
    x = _f64(x)
    y = np.empty_like(x)
    lib().dto_cube_operator(n, _p(slots), _p(lap), _p(areas), _p(kd), D(dt), _p(x), _p(y))
    return y


def cube_vcycle(n, slots, lap, areas, kd, dt, r):
    slots, lap, areas, kd = _cube_args(n, slots, lap, areas, kd)
    r = _f64(r)
    z = np.empty_like(r)
    lib().dto_cube_vcycle(n, _p(slots), _p(lap), _p(areas), _p(kd), D(dt), _p(r), _p(z))
    return z


def cube_lod(n, slots, lap, areas, kd, dt, h):
    slots, lap, areas, kd = _cube_args(n, slots, lap, areas, kd)
    h = _f64(h)
    x = np.empty_like(h)
    lib().dto_cube_lod(n, _p(slots), _p(lap), _p(areas), _p(kd), D(dt), _p(h), _p(x))
    return x


def cube_diff_solve(n, slots, lap, areas, kd, dt, tol_m, h):
    """surface/cube/diffusion.rs::solve with DiffusionSolver::Multigrid; returns (h', iterations)."""
    slots, lap, areas, kd = _cube_args(n, slots, lap, areas, kd)
    h = _f64(h).copy()
    its = lib().dto_cube_diff_solve(n, _p(slots), _p(lap), _p(areas), _p(kd), D(dt), D(tol_m), _p(h))
    return h, its


def diff_operator(x, kd, dt, dx, wrap=True):
    h, w = x.shape
    x, kd = _f64(x), _f64(kd)
    y = np.empty_like(x)
    lib().dto_diff_operator(w, h, D(dx), int(wrap), _p(kd), D(dt), _p(x), _p(y))
    return y


def diff_operator_coeffs(kd, dt, dx, wrap=True):
    h, w = kd.shape
    kd = _f64(kd)
    e, s, g = np.empty_like(kd), np.empty_like(kd), np.empty_like(kd)
    lib().dto_diff_operator_coeffs(w, h, D(dx), int(wrap), _p(kd), D(dt), _p(e), _p(s), _p(g))
    return e, s, g


def diff_apply_reference(x, kd, dt, dx, wrap=True):
    h, w = x.shape
    x, kd = _f64(x), _f64(kd)
    y = np.empty_like(x)
    lib().dto_diff_apply_reference(w, h, D(dx), int(wrap), _p(kd), D(dt), _p(x), _p(y))
    return y


def diff_lod(hfield, kd, dt, dx, wrap=True):
    x = _f64(hfield).copy()
    h, w = x.shape
    lib().dto_diff_lod(w, h, D(dx), int(wrap), _p(x), _p(_f64(kd)), D(dt))
    return x


def thomas(lo, di, up, b):
    b = _f64(b).copy()
    lib().dto_thomas(_p(_f64(lo)), _p(_f64(di)), _p(_f64(up)), _p(b), len(b))
    return b


def cyclic(lo, di, up, alpha, beta, b):
    b = _f64(b).copy()
    lib().dto_cyclic(_p(_f64(lo)), _p(_f64(di)), _p(_f64(up)), D(alpha), D(beta), _p(b), len(b))
    return b


def diff_solve_jacobi(hfield, kd, dt, dx, wrap=True, use_lod=True):
    """The reference's diffusion::step (Jacobi PCG to an RMS residual of 1e-6 m)."""
    x = _f64(hfield).copy()
    h, w = x.shape
    its = lib().dto_diff_solve_jacobi(w, h, D(dx), int(wrap), _p(x), _p(_f64(kd)), D(dt), int(use_lod))
    return x, its


def diff_solve_mg(hfield, kd, dt, dx, tol, wrap=True, stop=STOP_RMS_RESIDUAL, cycle=CYCLE_JACOBI, precision=32,
                  use_lod=True, max_it=400):
    """The reference's multigrid diffusion solve (diffusion::solve, Multigrid); returns
    (h', iterations, final relative residual ||b - A h'|| / ||b||)."""
    x = _f64(hfield).copy()
    h, w = x.shape
    rel = ctypes.c_double(0)
    its = lib().dto_diff_solve_mg(w, h, D(dx), int(wrap), _p(x), _p(_f64(kd)), D(dt), D(tol), stop, cycle, precision,
                                  int(use_lod), max_it, ctypes.byref(rel))
    return x, its, rel.value


def diff_vcycle(r, kd, dt, dx, wrap=True, cycle=CYCLE_JACOBI):
    h, w = r.shape
    r = _f64(r)
    z = np.empty((h, w), dtype=np.float32)
    nl = ctypes.c_int(0)
    rz = lib().dto_diff_vcycle(w, h, D(dx), int(wrap), _p(_f64(kd)), D(dt), cycle, _p(r), _p(z), ctypes.byref(nl))
    return z, rz, nl.value


def diff_reference_cg(b, kd, dt, dx, wrap=True, rel=1e-13):
    h, w = b.shape
    b = _f64(b)
    x = np.empty_like(b)
    lib().dto_diff_reference_cg(w, h, D(dx), int(wrap), _p(b), _p(_f64(kd)), D(dt), D(rel), _p(x))
    return x


def submarine_kd(z, d0, wave_base, tidal_range, land):
    return lib().dto_submarine_kd(z, d0, wave_base, tidal_range, land)
