"""Loads libdeeptime_gpu.so (built in-tree beside csrc/) and declares its C ABI
(include/deeptime_gpu.h). There is no CPU fallback: a missing library or device raises."""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libdeeptime_gpu.so")

DT_OK, DT_NOT_CONVERGED, DT_NONFINITE, DT_OOM, DT_BAD_ARG, DT_DEVICE_ERROR, DT_UNSUPPORTED = range(7)
STATUS_NAMES = {0: "DT_OK", 1: "DT_NOT_CONVERGED", 2: "DT_NONFINITE", 3: "DT_OOM", 4: "DT_BAD_ARG", 5: "DT_DEVICE_ERROR",
                6: "DT_UNSUPPORTED"}
PRECOND_REFERENCE, PRECOND_MEAN_D = 0, 1
STOP_MAX_Z, STOP_REL_RESIDUAL, STOP_RMS_RESIDUAL = 0, 1, 2
PREC_FP64, PREC_MIXED, PREC_MIXED_RELIABLE = 0, 1, 2
WARM_NONE, WARM_GIVEN, WARM_UNET = 0, 1, 2
CYCLE_JACOBI, CYCLE_RBGS = 0, 1
DIFF_FP64_CG_FP32_CYCLE, DIFF_FP64, DIFF_MIXED, DIFF_MIXED_RELIABLE = 0, 1, 2, 3


class FlexParams(ctypes.Structure):
    _fields_ = [("precond", ctypes.c_int), ("stop", ctypes.c_int), ("precision", ctypes.c_int),
                ("warm_start", ctypes.c_int), ("tol", ctypes.c_double), ("max_iterations", ctypes.c_int),
                ("inner_tol", ctypes.c_double), ("max_refinements", ctypes.c_int),
                ("host_loop", ctypes.c_int)]


class Report(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("error_m", ctypes.c_double), ("converged", ctypes.c_int),
                ("rel_residual", ctypes.c_double), ("refinements", ctypes.c_int),
                ("warm_start_accepted", ctypes.c_int), ("warm_start_rel_residual", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("kernel_launches", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DeepTimeError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DeepTimeError(DT_DEVICE_ERROR, f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.dt_last_error.restype = ctypes.c_char_p
        L.dt_device_info.argtypes = [ctypes.c_char_p, i]
        L.dt_flex_default_params.argtypes = [ctypes.POINTER(FlexParams)]
        L.dt_flex_create.argtypes = [i, i, d, vp, vp, ctypes.POINTER(vp)]
        L.dt_flex_destroy.argtypes = [vp]
        L.dt_flex_set_stream.argtypes = [vp, vp]
        for name in ("dt_flex_solve", "dt_flex_solve_dev"):
            getattr(L, name).argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(FlexParams), ctypes.POINTER(Report)]
        L.dt_flex_operator.argtypes = [vp, vp, vp, vp, vp]
        L.dt_flex_bend.argtypes = [vp, vp, vp, vp]
        L.dt_flex_precondition.argtypes = [vp, vp, vp, vp, vp, i, i]
        L.dt_flex_profile_kernels.argtypes = [vp, i, i, vp, vp]
        L.dt_flex_set_unet.argtypes = [vp, vp, d]
        L.dt_flex_operator_dot_noalloc.argtypes = [i, i, d, vp, vp, vp, vp, vp, vp]
        L.dt_cube_create.argtypes = [i, vp, vp, vp, ctypes.POINTER(vp)]
        L.dt_cube_destroy.argtypes = [vp]
        L.dt_cube_set_stream.argtypes = [vp, vp]
        L.dt_cube_levels.argtypes = [vp]
        for name in ("dt_cube_diff_solve", "dt_cube_diff_solve_dev"):
            getattr(L, name).argtypes = [vp, vp, vp, d, d, ctypes.POINTER(Report)]
        for name in ("dt_cube_operator", "dt_cube_vcycle", "dt_cube_lod"):
            getattr(L, name).argtypes = [vp, vp, d, vp, vp]
        L.dt_grid_restrict_dev.argtypes = [i, i, i, vp, vp, vp]
        L.dt_grid_prolong_const_dev.argtypes = [i, i, i, vp, vp, vp]
        L.dt_grid_prolong_linear_dev.argtypes = [i, i, i, vp, vp, vp]
        L.dt_grid_binomial_dev.argtypes = [i, i, i, vp, vp, vp]
        L.dt_grid_box_blur_dev.argtypes = [i, i, i, i, i, vp, vp, vp]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().dt_last_error().decode(errors="replace")


def check(status: int, allow=(DT_OK,)):
    if status not in allow:
        raise DeepTimeError(status, last_error())
    return status


def device_info() -> str | None:
    buf = ctypes.create_string_buffer(256)
    ok = lib().dt_device_info(buf, 256)
    return buf.value.decode() if ok else None
