"""Shared seeded inputs and parameter sets for the parity tests."""
from __future__ import annotations

import functools
import itertools

import numpy as np

from polyspectrum_b200 import synth

FIELD_NAMES = {0: "DENS", 1: "XHII", 2: "XHI_DENS"}


@functools.lru_cache(maxsize=None)
def fields(n: int, box: float, seed: int = 1):
    """(dens, xhii) float32 grids: lognormal density (k^-2) and ionised spheres."""
    dens = synth.lognormal_density(n, 2.0, seed)
    count = max(8, int(round(40 * (n / 16) ** 3 / 8)))
    xhii = synth.ionised_spheres(n, box, count, seed + 1, median_radius=box / n * 2.0)
    return dens, xhii


def field_args(which: int, dens, xhii):
    """(dens, xhii) as get_FT_field consumes them for `which`."""
    if which == 0:
        return dens, None
    if which == 1:
        return None, xhii
    return (1.0 + dens.astype(np.float64)).astype(np.float32), xhii


def sweep_params(n_grid: int, box: float):
    """A matrix of run parameters covering every binning case, n = 2 and 3,
    equilateral and theta sweeps, phase on and off, and the three fields."""
    kf = 2 * np.pi / box
    out = []
    for kb, phase, which in itertools.product((0, 1, 2, 3), (0, 1), (0, 1, 2)):
        # theta sweep with legs of a few fundamental modes
        out.append(dict(n=3, equilateral=0, k1=3.2 * kf, k2=4.6 * kf, num_values=6, theta=0.5,
                        kbinwidth=1.0, kbinning=kb, dcos_theta=0.2, use_only_phase=phase,
                        which_field=which))
        # equilateral sweep
        out.append(dict(n=3, equilateral=1, k1=0.0, k2=0.0, num_values=4, theta=0.0,
                        kbinwidth=1.0, kbinning=kb, dcos_theta=0.2, use_only_phase=phase,
                        which_field=which))
        if kb != 1:  # n=2 DERIVED is undefined in the reference (filter.c:321-325)
            out.append(dict(n=2, equilateral=0, k1=0.0, k2=0.0, num_values=2, theta=0.0,
                            kbinwidth=1.0, kbinning=kb, dcos_theta=0.2, use_only_phase=phase,
                            which_field=which))
    return out


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), 1e-300)
    return np.abs(a - b) / den
