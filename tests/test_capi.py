"""The C ABI without a GPU: the library loads, exports every entry point include/ declares, and
rejects bad arguments before touching a device."""
import ctypes
import os
import re

import pytest

from deeptime_gpu import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if fn.endswith(".h"):
            text = open(os.path.join(HEADER_DIR, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names.update(re.findall(r"\b(dt_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(L.LIB_PATH):
        import subprocess

        subprocess.run(["make", "-s", "-C", L.PKG_DIR], check=True)
    return L.lib()


def test_every_declared_entry_point_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bad_shapes_are_rejected_before_any_device_work(lib):
    h = ctypes.c_void_p()
    assert lib.dt_flex_create(0, 8, 1000.0, None, None, ctypes.byref(h)) == L.DT_BAD_ARG
    assert lib.dt_flex_create(16, 8, -1.0, None, None, ctypes.byref(h)) == L.DT_BAD_ARG
    # any width up to 65536 and any height up to 8192: past those, refused before the device
    assert lib.dt_flex_create(70000, 8, 1000.0, None, None, ctypes.byref(h)) == L.DT_UNSUPPORTED
    assert "65536" in L.last_error()
    assert lib.dt_flex_create(16, 9000, 1000.0, None, None, ctypes.byref(h)) == L.DT_UNSUPPORTED
    assert lib.dt_flex_create(16, 8, 1000.0, None, None, None) == L.DT_BAD_ARG


def test_default_params_are_the_references(lib):
    p = L.FlexParams()
    lib.dt_flex_default_params(ctypes.byref(p))
    # FlexureParams::default: tolerance 2 m, 60 iterations (flexure.rs:224-225); the reference
    # preconditioner and stopping rule; FP64
    assert (p.tol, p.max_iterations, p.precond, p.stop, p.precision) == (2.0, 60, L.PRECOND_REFERENCE, L.STOP_MAX_Z,
                                                                           L.PREC_FP64)


def test_no_device_means_an_error_not_a_fallback(lib):
    if L.device_info() is not None:
        pytest.skip("a CUDA device is present")
    h = ctypes.c_void_p()
    assert lib.dt_flex_create(16, 8, 1000.0, None, None, ctypes.byref(h)) == L.DT_DEVICE_ERROR
