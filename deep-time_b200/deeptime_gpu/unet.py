"""The learned warm start for the flexure solve: data, training and prediction.

The network and its training are the library's (dt_unet_* in include/deeptime_gpu.h: tensor-core
convolution kernels, Adam, MSE). This module supplies the data and the loop:

  inputs   x0 = b / rms(b), x1 = (log10(d g) - 22.5) / 1.5  (d = D/g, b = q/g of Solver::solve)
  target   w c / rms(b): the deflection over the local-isostasy scale q / (delta-rho g)

Training pairs follow the 512 x 256, dx = 10 km workload (rigidity smoothed over 8 cells, a |k|^-2
load field of std 1500 m), generated on the device with the same SplitMix64 streams as
inputs.flexure_problem, and labelled by this library's FP64 PCG to a relative residual of 1e-10.
torch holds the device memory and does the fields' FFT filtering (data plumbing).
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _lib as L
from . import flexure as F

G = 9.81
C_MANTLE = 3300.0
LOGD_MID, LOGD_HALF = 22.5, 1.5


def _declare(lib):
    if getattr(lib, "_unet_declared", False):
        return
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.dt_unet_create.argtypes = [i, ctypes.c_ulonglong, ctypes.POINTER(vp)]
    lib.dt_unet_destroy.argtypes = [vp]
    lib.dt_unet_num_params.argtypes = [vp]
    lib.dt_unet_num_params.restype = ctypes.c_size_t
    lib.dt_unet_set_stream.argtypes = [vp, vp]
    lib.dt_unet_predict_dev.argtypes = [vp, vp, vp, i, i, i]
    lib.dt_unet_train_step_dev.argtypes = [vp, vp, vp, i, i, i, ctypes.c_float, ctypes.POINTER(d)]
    lib.dt_unet_loss_and_grad_dev.argtypes = [vp, vp, vp, i, i, i, ctypes.POINTER(d)]
    for name in ("dt_unet_gradients", "dt_unet_get_params", "dt_unet_set_params"):
        getattr(lib, name).argtypes = [vp, vp, ctypes.c_size_t]
    lib.dt_unet_save.argtypes = [vp, ctypes.c_char_p]
    lib.dt_unet_load.argtypes = [vp, ctypes.c_char_p]
    lib._unet_declared = True


class UNet:
    """A handle on the library's U-Net (weights on the device)."""

    def __init__(self, seed: int = 12345):
        lib = L.lib()
        _declare(lib)
        h = ctypes.c_void_p()
        L.check(lib.dt_unet_create(32, seed, ctypes.byref(h)))
        self._h = h
        self.n_params = lib.dt_unet_num_params(h)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().dt_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        L.check(L.lib().dt_unet_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def predict_dev(self, x_ptr, y_ptr, B, H, W):
        L.check(L.lib().dt_unet_predict_dev(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), B, H, W))

    def train_step_dev(self, x_ptr, t_ptr, B, H, W, lr):
        loss = ctypes.c_double(0)
        L.check(L.lib().dt_unet_train_step_dev(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(t_ptr), B, H, W,
                                               ctypes.c_float(lr), ctypes.byref(loss)))
        return loss.value

    def loss_and_grad_dev(self, x_ptr, t_ptr, B, H, W):
        loss = ctypes.c_double(0)
        L.check(L.lib().dt_unet_loss_and_grad_dev(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(t_ptr), B, H, W,
                                                  ctypes.byref(loss)))
        return loss.value

    def _vec(self, name, arr=None):
        if arr is None:
            arr = np.empty(self.n_params, dtype=np.float32)
            L.check(getattr(L.lib(), name)(self._h, ctypes.c_void_p(arr.ctypes.data), self.n_params))
            return arr
        arr = np.ascontiguousarray(arr, dtype=np.float32)
        L.check(getattr(L.lib(), name)(self._h, ctypes.c_void_p(arr.ctypes.data), self.n_params))

    def gradients(self):
        return self._vec("dt_unet_gradients")

    def params(self):
        return self._vec("dt_unet_get_params")

    def set_params(self, p):
        self._vec("dt_unet_set_params", p)

    def save(self, path):
        L.check(L.lib().dt_unet_save(self._h, path.encode()))

    def load(self, path):
        L.check(L.lib().dt_unet_load(self._h, path.encode()))


# ---- data on the device ------------------------------------------------------------------------

GOLDEN, M1, M2 = 0x9E3779B97F4A7C15, 0xBF58476D1CE4E5B9, 0x94D049BB133111EB


def _s64(v):
    return v - (1 << 64) if v >= (1 << 63) else v


def _lsr(z, k):
    import torch

    return (z >> k) & ((1 << (64 - k)) - 1)


def splitmix_f64_torch(seed: int, n: int, device):
    """SplitMix64 next_f64 draws 1..n of SplitMix64(seed), bit-identical to inputs.splitmix64_f64."""
    import torch

    k = torch.arange(1, n + 1, dtype=torch.int64, device=device)
    z = k * _s64(GOLDEN) + _s64(seed & 0xFFFFFFFFFFFFFFFF)
    z = (z ^ _lsr(z, 30)) * _s64(M1)
    z = (z ^ _lsr(z, 27)) * _s64(M2)
    z = z ^ _lsr(z, 31)
    return _lsr(z, 11).to(torch.float64) * (1.0 / float(1 << 53))


def splitmix_normal_torch(seed, n, device):
    import torch

    f = splitmix_f64_torch(seed, 2 * n, device)
    u = torch.clamp(f[0::2], min=np.finfo(np.float64).tiny)
    return torch.sqrt(-2.0 * torch.log(u)) * torch.cos(2.0 * math.pi * f[1::2])


def _smooth(v, sigma):
    import torch

    h, w = v.shape
    ext = torch.cat([v, torch.flip(v, dims=[0])], dim=0)
    fy = torch.fft.fftfreq(2 * h, device=v.device, dtype=torch.float64)[:, None]
    fx = torch.fft.rfftfreq(w, device=v.device, dtype=torch.float64)[None, :]
    gain = torch.exp(-2.0 * (math.pi * sigma) ** 2 * (fx * fx + fy * fy))
    return torch.fft.irfft2(torch.fft.rfft2(ext) * gain, s=ext.shape)[:h]


def _grf(w, h, beta, std, seed, device):
    import torch

    noise = splitmix_normal_torch(seed, w * h, device).reshape(h, w)
    fy = torch.fft.fftfreq(h, device=device, dtype=torch.float64)[:, None]
    fx = torch.fft.rfftfreq(w, device=device, dtype=torch.float64)[None, :]
    k2 = fx * fx + fy * fy
    k2[0, 0] = 1.0
    amp = k2 ** (-beta / 4.0)
    amp[0, 0] = 0.0
    f = torch.fft.irfft2(torch.fft.rfft2(noise) * amp, s=(h, w))
    f = f - f.mean()
    s = f.std(unbiased=False)
    return f * (std / s)


def flexure_problem_torch(w, h, sigma, seed, device, topo_std=1500.0, beta=2.0):
    """inputs.flexure_problem on the device: (d, c, b) float64 tensors."""
    import torch

    u = _smooth(splitmix_normal_torch(seed, w * h, device).reshape(h, w), sigma)
    u = (u - u.min()) / (u.max() - u.min())
    D = 10.0 ** (21.0 + 3.0 * u)
    topo = _grf(w, h, beta, topo_std, seed + 1, device)
    return D / G, torch.full((h, w), C_MANTLE, dtype=torch.float64, device=device), 2700.0 * topo


def diffusion_problem_torch(w, h, sigma, seed, device, topo_std=800.0, beta=2.5):
    """inputs.diffusion_problem on the device: (h0, s) float64 tensors, s = kappa dt / dx^2 a
    smoothed log-uniform field over [0.1, 100]."""
    topo = _grf(w, h, beta, topo_std, seed, device)
    v = _smooth(splitmix_f64_torch(seed + 1, w * h, device).reshape(h, w), sigma)
    lo, hi = v.min(), v.max()
    v = (v - lo) / (hi - lo)
    return topo, 10.0 ** (-1.0 + 3.0 * v)


def normalise_inputs(d, b, c_mean=C_MANTLE):
    """(x [h][w][2] float32, scale) with scale = rms(b) / c_mean, so that w = prediction * scale."""
    import torch

    rms = torch.sqrt(torch.mean(b * b))
    x0 = b / rms
    x1 = (torch.log10(d * G) - LOGD_MID) / LOGD_HALF
    return torch.stack([x0, x1], dim=-1).to(torch.float32), float(rms) / c_mean


def make_dataset(n, w=512, h=256, dx=10_000.0, sigma=8.0, seed0=50_000, tol=1e-10, log=None):
    """n labelled pairs on the device: X [n][h][w][2], T [n][h][w] (float32), the labels' PCG
    iteration counts and relative residuals."""
    import torch

    dev = torch.device("cuda")
    X = torch.empty((n, h, w, 2), dtype=torch.float32, device=dev)
    T = torch.empty((n, h, w), dtype=torch.float32, device=dev)
    sv = F.Solver(w, h, dx)
    p = F.params(precond=L.PRECOND_REFERENCE, stop=L.STOP_REL_RESIDUAL, precision=L.PREC_FP64, tol=tol,
                 max_iterations=5000)
    lib = L.lib()
    x_dev = torch.zeros((h, w), dtype=torch.float64, device=dev)
    its, rels = [], []
    t0 = time.time()
    for k in range(n):
        d, c, b = flexure_problem_torch(w, h, sigma, seed0 + 2 * k, dev)
        torch.cuda.synchronize()
        rep = L.Report()
        st = lib.dt_flex_solve_dev(sv._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                   ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x_dev.data_ptr()), ctypes.byref(p),
                                   ctypes.byref(rep))
        L.check(st)
        xin, scale = normalise_inputs(d, b)
        X[k] = xin
        T[k] = (x_dev / scale).to(torch.float32)
        its.append(rep.iterations)
        rels.append(rep.rel_residual)
        if log and (k + 1) % 2000 == 0:
            log(f"  labelled {k + 1}/{n} in {time.time() - t0:.1f} s")
    sv.close()
    return X, T, its, rels


def train(model: UNet, X, T, epochs=50, batch=16, lr=1e-3, seed=7, log=None):
    """Adam on MSE over shuffled mini-batches; returns the mean loss of each epoch."""
    import torch

    n, h, w = T.shape
    rng = np.random.default_rng(seed)
    history = []
    for ep in range(epochs):
        order = torch.from_numpy(rng.permutation(n)).to(X.device)
        tot, cnt = 0.0, 0
        t0 = time.time()
        for s in range(0, n - batch + 1, batch):
            idx = order[s:s + batch]
            xb = X.index_select(0, idx).contiguous()
            tb = T.index_select(0, idx).contiguous()
            tot += model.train_step_dev(xb.data_ptr(), tb.data_ptr(), batch, h, w, lr)
            cnt += 1
        history.append(tot / max(cnt, 1))
        if log:
            log(f"  epoch {ep + 1}/{epochs}: loss {history[-1]:.5f} ({time.time() - t0:.1f} s)")
    return history


def predict(model: UNet, X):
    import torch

    n, h, w, _ = X.shape
    Y = torch.empty((n, h, w), dtype=torch.float32, device=X.device)
    for k in range(n):
        model.predict_dev(X[k].data_ptr(), Y[k].data_ptr(), 1, h, w)
    return Y
