"""Seeded synthetic inputs for the flexure and diffusion solves (numpy, host side).

Random numbers come from SplitMix64 (Steele, Lea & Flood 2014), the generator the reference seeds
its tests with (crates/deeptime-core/src/sphere/mod.rs:43-80): `next_u64`, `next_f64` (53 bits)
and Box-Muller `normal`, here vectorised: the k-th call's state is seed + k * 0x9E3779B97F4A7C15.

The fields follow the benchmark workloads' recipes:
  - rigidity: white N(0,1) noise, Gaussian-smoothed (sigma cells; x wraps, y reflects), rescaled
    to [0, 1] as u, D = 10^(21 + 3u) N m;
  - topography: a Gaussian random field with power spectrum ~ |k|^-beta, zero mean, given std;
  - load q = 2700 * 9.81 * h, restoring density 3300 kg/m^3.
The flexure solve takes d = D/g, c = delta-rho, b = q/g (units of the reference's
Solver::solve, crates/deeptime-core/src/surface/flexure.rs:1677-1679).
"""
from __future__ import annotations

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)
G = 9.81
RHO_CRUST_LOAD = 2700.0
RHO_MANTLE = 3300.0


def splitmix64_u64(seed: int, n: int, start: int = 0) -> np.ndarray:
    """The next_u64 values of calls start+1 .. start+n of SplitMix64(seed)."""
    k = np.arange(start + 1, start + n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * GOLDEN
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return z


def splitmix64_f64(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Uniform [0, 1) with 53 bits, as SplitMix64::next_f64."""
    return (splitmix64_u64(seed, n, start) >> np.uint64(11)).astype(np.float64) * (1.0 / float(1 << 53))


def splitmix64_normal(seed: int, n: int) -> np.ndarray:
    """n standard normal deviates, as n successive SplitMix64::normal calls (Box-Muller, two draws
    per deviate)."""
    f = splitmix64_f64(seed, 2 * n)
    u = np.maximum(f[0::2], np.finfo(np.float64).tiny)
    v = f[1::2]
    return np.sqrt(-2.0 * np.log(u)) * np.cos(2.0 * np.pi * v)


class SplitMix64:
    """The sequential generator, for the few draws the small test fixtures take."""

    def __init__(self, seed: int):
        self.state = seed & 0xFFFFFFFFFFFFFFFF

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    def next_f64(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / float(1 << 53))


def gaussian_smooth(v: np.ndarray, sigma: float) -> np.ndarray:
    """Gaussian blur with standard deviation `sigma` cells, x periodic and y reflecting (the field
    is mirrored about its first and last row edges and the convolution taken by FFT)."""
    h, w = v.shape
    ext = np.concatenate([v, v[::-1]], axis=0)
    fy = np.fft.fftfreq(2 * h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    gain = np.exp(-2.0 * (np.pi * sigma) ** 2 * (fx * fx + fy * fy))
    out = np.fft.irfft2(np.fft.rfft2(ext) * gain, s=ext.shape)
    return out[:h]


def gaussian_random_field(w: int, h: int, beta: float, std: float, seed: int) -> np.ndarray:
    """Zero-mean field with power spectrum ~ |k|^-beta (white noise filtered by |k|^(-beta/2), the
    k = 0 term removed), scaled to the given standard deviation."""
    noise = splitmix64_normal(seed, w * h).reshape(h, w)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    k2 = fx * fx + fy * fy
    k2[0, 0] = 1.0
    amp = k2 ** (-beta / 4.0)
    amp[0, 0] = 0.0
    f = np.fft.irfft2(np.fft.rfft2(noise) * amp, s=(h, w))
    f -= f.mean()
    s = f.std()
    return f * (std / s) if s > 0 else f


def rigidity_field(w: int, h: int, sigma: float, seed: int) -> np.ndarray:
    """D = 10^(21 + 3u), u the smoothed white noise rescaled to [0, 1]."""
    u = gaussian_smooth(splitmix64_normal(seed, w * h).reshape(h, w), sigma)
    lo, hi = u.min(), u.max()
    u = (u - lo) / (hi - lo) if hi > lo else np.zeros_like(u)
    return 10.0 ** (21.0 + 3.0 * u)


def flexure_problem(w: int, h: int, sigma: float, seed: int, topo_std: float = 1500.0, beta: float = 2.0):
    """(d, c, b) for Solver::solve: d = D/g, c = 3300, b = q/g = 2700 h, with the rigidity seeded
    by `seed` and the topography by `seed + 1`."""
    D = rigidity_field(w, h, sigma, seed)
    topo = gaussian_random_field(w, h, beta, topo_std, seed + 1)
    d = D / G
    c = np.full((h, w), RHO_MANTLE)
    b = RHO_CRUST_LOAD * G * topo / G
    return d, c, b


def diffusion_problem(w: int, h: int, sigma: float, seed: int, topo_std: float = 800.0, beta: float = 2.5):
    """(h0, s) for the implicit diffusion solve: h0 a |k|^-2.5 field of std 800 m and
    s = kappa dt / dx^2 = 10^(-1 + 3v), v the smoothed uniform noise rescaled to [0, 1] (a
    log-uniform field over [0.1, 100])."""
    topo = gaussian_random_field(w, h, beta, topo_std, seed)
    v = gaussian_smooth(splitmix64_f64(seed + 1, w * h).reshape(h, w), sigma)
    lo, hi = v.min(), v.max()
    v = (v - lo) / (hi - lo) if hi > lo else np.zeros_like(v)
    s = 10.0 ** (-1.0 + 3.0 * v)
    return topo, s


def cube_problem(n: int, seed: int, slots: np.ndarray):
    """(lap, areas, kd, h) for the cube grid's diffusion on `slots` (cube.topology(n)): cell
    areas within 20% of each other; coupling weights symmetric across every pair, as
    CubeGrid::lap is (each pair takes the value its lower-indexed cell computed,
    sphere/cube.rs:300-316), side pairs near 1 and diagonal pairs small; a diffusivity field with
    a sharp land-sea edge; h of std 1000 m. Seeded by numpy's default generator."""
    rng = np.random.default_rng(seed)
    cells = 6 * n * n
    areas = 1.0 + 0.2 * rng.random(cells)
    raw = np.where(np.arange(8) % 2 == 0, 0.8 + 0.4 * rng.random((cells, 8)), 0.05 + 0.15 * rng.random((cells, 8)))
    valid = slots != 0xFFFFFFFF
    m = np.where(valid, slots, 0).astype(np.int64)
    c = np.arange(cells)[:, None]
    back = np.argmax(slots[m] == c[:, :, None], axis=2)  # the slot of c in its neighbour m's table
    lap = np.where(m > c, raw, raw[m, back])
    lap = np.where(valid, lap, 0.0)
    kd = np.where(rng.random(cells) < 0.3, 0.02, 1.0) * (0.5 + rng.random(cells))
    h = 1000.0 * rng.standard_normal(cells)
    return lap, areas, kd, h
