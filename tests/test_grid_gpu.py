"""The step's grid helpers on the device (restrict, prolong, binomial, box blur) against the
oracle's restatement of the reference, through the C ABI. The bar is bit-for-bit: every one of
them is the reference's arithmetic in the reference's order."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from deeptime_gpu import _lib as L

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


SIZES = [(8, 8), (64, 32), (37, 19), (256, 128), (1024, 328)]


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("f", [1, 2, 3, 4])
def test_restrict_and_prolong_are_the_references(w, h, f):
    if w // f < 1 or h // f < 1:
        pytest.skip("raster smaller than a block")
    rng = np.random.default_rng(w * 31 + h + f)
    v = rng.standard_normal((h, w)) * 1e3
    lib = L.lib()
    fine = dev(v)
    coarse = torch.empty((h // f, w // f), dtype=torch.float64, device="cuda")
    L.check(lib.dt_grid_restrict_dev(w, h, f, ptr(fine), ptr(coarse), None))
    want = O.restrict_by(v, f)
    got = host(coarse)
    assert np.array_equal(got, want)
    back = torch.empty(((h // f) * f, (w // f) * f), dtype=torch.float64, device="cuda")
    L.check(lib.dt_grid_prolong_const_dev(w // f, h // f, f, ptr(coarse), ptr(back), None))
    assert np.array_equal(host(back), O.prolong_const(want, f))
    L.check(lib.dt_grid_prolong_linear_dev(w // f, h // f, f, ptr(coarse), ptr(back), None))
    assert np.array_equal(host(back), O.prolong_linear(want, f))


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("passes", [0, 1, 3])
def test_binomial_is_the_references(w, h, passes):
    rng = np.random.default_rng(w + 7 * h + passes)
    v = rng.standard_normal((h, w))
    t, s = dev(v), torch.empty((h, w), dtype=torch.float64, device="cuda")
    L.check(L.lib().dt_grid_binomial_dev(w, h, passes, ptr(t), ptr(s), None))
    assert np.array_equal(host(t), O.binomial(v, passes))


@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("r,passes", [(1, 2), (2, 2), (3, 1), (0, 2), (31, 1), (40, 1), (63, 1), (70, 1)])
@pytest.mark.parametrize("wrap", [True, False])
def test_box_blur_is_the_references(w, h, r, passes, wrap):
    # r up to 31 and up to 63: the line kernel's two window widths; 70: the plain kernels
    rng = np.random.default_rng(w + 11 * h + r)
    v = rng.standard_normal((h, w)) * 50.0 + 25.0
    t, s = dev(v), torch.empty((h, w), dtype=torch.float64, device="cuda")
    L.check(L.lib().dt_grid_box_blur_dev(w, h, int(wrap), r, passes, ptr(t), ptr(s), None))
    assert np.array_equal(host(t), O.box_blur(v, r, passes, wrap=wrap))


def test_bad_arguments_are_refused():
    lib = L.lib()
    t = dev(np.zeros((4, 4)))
    assert lib.dt_grid_restrict_dev(4, 4, 8, ptr(t), ptr(t), None) == L.DT_BAD_ARG
    assert lib.dt_grid_prolong_linear_dev(0, 4, 2, ptr(t), ptr(t), None) == L.DT_BAD_ARG
    assert lib.dt_grid_binomial_dev(4, 4, 1, ptr(t), None, None) == L.DT_BAD_ARG
    assert lib.dt_grid_box_blur_dev(4, 4, 1, -1, 1, ptr(t), ptr(t), None) == L.DT_BAD_ARG


def test_the_python_mirror_runs_the_same_kernels():
    from deeptime_gpu import grid as Gr

    rng = np.random.default_rng(9)
    v = rng.standard_normal((64, 96)) * 10.0
    c = Gr.restrict(dev(v), 4)
    assert np.array_equal(host(c), O.restrict_by(v, 4))
    assert np.array_equal(host(Gr.prolong_linear(c, 4)), O.prolong_linear(O.restrict_by(v, 4), 4))
    assert np.array_equal(host(Gr.prolong_const(c, 4)), O.prolong_const(O.restrict_by(v, 4), 4))
    assert np.array_equal(host(Gr.binomial(dev(v), 2)), O.binomial(v, 2))
    assert np.array_equal(host(Gr.box_blur(dev(v), 2, 2, wrap_x=False)), O.box_blur(v, 2, 2, wrap=False))
