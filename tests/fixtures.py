"""Small seeded fixtures restated from the reference's tests (no GPU, no oracle calls)."""
import numpy as np

from deeptime_gpu.inputs import SplitMix64


def terrain(w, h, seed):
    """A few octaves of value noise, metres (multigrid/tests.rs:77-98)."""
    rng = SplitMix64(seed)
    z = np.zeros((h, w))
    j = np.arange(h)[:, None].astype(np.float64)
    i = np.arange(w)[None, :].astype(np.float64)
    for oct in range(6):
        g = 2 << oct
        grid = np.array([rng.next_f64() - 0.5 for _ in range(g * g)])
        amp = 3000.0 / float(1 << oct)
        fy = j / max(h, 1) * (g - 1)
        j0 = np.floor(fy).astype(np.int64)
        ty = fy - j0
        fx = i / w * g
        i0 = np.floor(fx).astype(np.int64)
        tx = fx - i0

        def at(a, b):
            return grid[np.minimum(b, g - 1) * g + a % g]

        top = at(i0, j0) * (1.0 - tx) + at(i0 + 1, j0) * tx
        bot = at(i0, j0 + 1) * (1.0 - tx) + at(i0 + 1, j0 + 1) * tx
        z += amp * (top * (1.0 - ty) + bot * ty)
    return z


def submarine_kd(z, d0, wave_base, tidal_range, land):
    """Landlab's SimpleSubmarineDiffuser diffusivity (marine.rs:44-59), vectorised."""
    if tidal_range > 0.0:
        f1 = (np.tanh(z / tidal_range) + 1.0) / 2.0
    else:
        f1 = np.where(z >= 0.0, 1.0, 0.0)
    if wave_base > 0.0:
        f2 = np.where(z > wave_base, np.exp(-(z - wave_base) / wave_base), 1.0)
    else:
        f2 = np.ones_like(z)
    return d0 * f1 * f2 + land * (1.0 - f1)


def shelf_kd(z, seed):
    """The surface stage's diffusivities on z (multigrid/tests.rs:102-110)."""
    rng = SplitMix64(seed ^ 0x5EED)
    land = np.array([2.0 * (0.25 + 4.0 * rng.next_f64()) for _ in range(z.size)]).reshape(z.shape)
    return submarine_kd(-z, 100.0, 60.0, 2.0, land)


def diffusion_bound(east, south, diag, tol):
    """multigrid/tests.rs:157-164: the RMS error a solve stopped at an RMS residual of tol may have."""
    n = diag.size
    g1 = diag - 1.0
    mean = g1.sum() / n
    rms = np.sqrt((g1 * g1).sum() / n)
    return tol * (1.0 + (rms / mean if mean > 0 else 0.0)) * 1.01


def rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2))) if a.size else 0.0


SIZES = [(1, 1), (1, 7), (7, 1), (2, 2), (2, 5), (3, 5), (5, 3), (17, 9), (33, 33), (64, 40), (129, 67), (200, 96)]


def cube_case(n, seed, slots):
    """A seeded cube-grid geometry for the cube diffusion's parity tests (the package's
    inputs.cube_problem): cell areas within 20% of each other, symmetric coupling weights (side
    pairs near 1, diagonal pairs small), a diffusivity field with a sharp land-sea edge."""
    from deeptime_gpu import inputs as I

    return I.cube_problem(n, seed, slots)
