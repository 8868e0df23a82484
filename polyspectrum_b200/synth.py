"""Seeded synthetic input grids.

The reference reads raw row-major float32/float64 grids (grid.c:122-228) that
are not shipped with it; these generators stand in for them with the shapes,
sizes and value distributions of the reference's use cases:

* ``gaussian_field``: white noise -> rFFT -> times sqrt(P(k)), P ~ k^-alpha for
  0 < |k| <= k_Nyquist and 0 elsewhere -> irFFT -> rescaled to unit variance.
* ``lognormal_density``: delta = exp(g - var/2) - 1 for a Gaussian field g.
* ``ionised_spheres``: binary x_HII map, 1 inside any of ``count`` spheres with
  uniform centres and lognormal radii (median 3 Mpc/h, sigma_ln 0.5), periodic.

All outputs are float32 arrays of shape (N, N, N), C order (the reference's
[i][j][l] layout).
"""
from __future__ import annotations

import numpy as np

try:
    import scipy.fft as _fft

    def _rfftn(a):
        return _fft.rfftn(a, workers=-1)

    def _irfftn(a, s):
        return _fft.irfftn(a, s=s, workers=-1)

except ImportError:  # pragma: no cover
    def _rfftn(a):
        return np.fft.rfftn(a)

    def _irfftn(a, s):
        return np.fft.irfftn(a, s=s)


def gaussian_field(n: int, alpha: float, seed: int) -> np.ndarray:
    """Unit-variance Gaussian random field with P(k) ~ k^-alpha up to Nyquist."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((n, n, n), dtype=np.float32)
    wk = _rfftn(white)
    f = np.fft.fftfreq(n).astype(np.float32) * n
    fz = np.fft.rfftfreq(n).astype(np.float32) * n
    k2 = f[:, None, None] ** 2 + f[None, :, None] ** 2 + fz[None, None, :] ** 2
    kk = np.sqrt(k2)
    amp = np.zeros_like(kk)
    nz = (kk > 0) & (kk <= n / 2)
    amp[nz] = kk[nz] ** (-alpha / 2.0)
    wk *= amp
    g = _irfftn(wk, s=(n, n, n)).astype(np.float32)
    g -= g.mean(dtype=np.float64)
    g /= np.float32(np.sqrt(g.var(dtype=np.float64)))
    return g


def lognormal_density(n: int, alpha: float, seed: int) -> np.ndarray:
    """delta = exp(g - var/2) - 1 (var(g) = 1), float32."""
    g = gaussian_field(n, alpha, seed)
    return (np.exp(g.astype(np.float64) - 0.5) - 1.0).astype(np.float32)


def ionised_spheres(n: int, box: float, count: int, seed: int,
                    median_radius: float = 3.0, sigma_ln: float = 0.5) -> np.ndarray:
    """Binary x_HII grid: voxel centres inside any periodic sphere are 1."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, box, size=(count, 3))
    radii = median_radius * np.exp(sigma_ln * rng.standard_normal(count))
    cell = box / n
    out = np.zeros((n, n, n), dtype=np.float32)
    for c, r in zip(centres, radii):
        lo = np.floor((c - r) / cell - 0.5).astype(np.int64)
        hi = np.ceil((c + r) / cell - 0.5).astype(np.int64)
        axes = []
        for d in range(3):
            idx = np.arange(lo[d], hi[d] + 1)
            pos = (idx + 0.5) * cell - c[d]
            axes.append((np.mod(idx, n), pos * pos))
        (ix, dx), (iy, dy), (iz, dz) = axes
        inside = (dx[:, None, None] + dy[None, :, None] + dz[None, None, :]) <= r * r
        if not inside.any():
            continue
        sub = out[np.ix_(ix, iy, iz)]
        sub[inside] = 1.0
        out[np.ix_(ix, iy, iz)] = sub
    return out


def xhi_dens_inputs(n: int, box: float, count: int, seed_ion: int, alpha: float,
                    seed_dens: int) -> tuple[np.ndarray, np.ndarray]:
    """(density file = 1 + delta, ion file = x_HII) whose product field is
    dens*(1 - xHII), as input_field.c:33 forms it."""
    dens = (1.0 + lognormal_density(n, alpha, seed_dens).astype(np.float64)).astype(np.float32)
    xhii = ionised_spheres(n, box, count, seed_ion)
    return dens, xhii
