"""Generate the golden fixtures of this directory from the UNMODIFIED reference.

    make -C oracle ref            # builds oracle/_ref/libpsref.so from the reference sources
    python tests/golden/make_golden.py

Inputs are seeded synthetic grids (polyspectrum_b200/synth.py) stored as raw
float32 files next to the JSON, so the fixtures do not depend on the FFT used
to synthesise them.  Each JSON holds one run of the reference (run.c:56-92
through oracle/ref_harness.c): the sweep values and, per configuration, B,
Npolygons and the kpolygon / kpolygonMin / kpolygonMax arrays after the call,
all as exact doubles.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from polyspectrum_b200 import synth  # noqa: E402


def write_raw(name: str, a: np.ndarray) -> str:
    np.ascontiguousarray(a, dtype=np.float32).tofile(os.path.join(HERE, name))
    return name


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libpsref.so missing: run `make -C oracle ref` first")
    cases = []
    for n, box in ((16, 100.0), (32, 200.0)):
        dens = synth.lognormal_density(n, 2.0, 11)
        xhii = synth.ionised_spheres(n, box, 6 if n == 16 else 40, 12, median_radius=box / n * 2.0)
        dens1p = (1.0 + dens.astype(np.float64)).astype(np.float32)
        fd = write_raw(f"dens_N{n}.f32", dens)
        fx = write_raw(f"xhii_N{n}.f32", xhii)
        f1 = write_raw(f"dens1p_N{n}.f32", dens1p)
        kf = 2 * np.pi / box
        base = dict(grid_size=n, box_size=box, kbinwidth=1.0, dcos_theta=0.2, write_numpolygons=1)
        cases += [
            (f"N{n}_dens_sweep_default", fd, None,
             dict(base, which_field=0, n=3, equilateral=0, k1=3.1 * kf, k2=4.4 * kf,
                  num_values=6, kbinning=0)),
            (f"N{n}_dens_sweep_derived", fd, None,
             dict(base, which_field=0, n=3, equilateral=0, k1=3.1 * kf, k2=4.4 * kf,
                  num_values=6, kbinning=1)),
            (f"N{n}_xhii_sweep_given", None, fx,
             dict(base, which_field=1, n=3, equilateral=0, k1=2.6 * kf, k2=3.9 * kf,
                  num_values=5, kbinning=2)),
            (f"N{n}_dens_sweep_watkinson", fd, None,
             dict(base, which_field=0, n=3, equilateral=0, k1=3.1 * kf, k2=4.4 * kf,
                  num_values=4, kbinning=3)),
            (f"N{n}_dens_equilateral", fd, None,
             dict(base, which_field=0, n=3, equilateral=1, num_values=5, kbinning=0)),
            (f"N{n}_dens_power", fd, None,
             dict(base, which_field=0, n=2, num_values=2, kbinning=0)),
            (f"N{n}_xhidens_phase_derived", f1, fx,
             dict(base, which_field=2, use_only_phase=1, n=3, equilateral=0, k1=2.2 * kf,
                  k2=3.4 * kf, num_values=6, kbinning=1)),
        ]
    for name, fd, fx, params in cases:
        n = params["grid_size"]
        load = lambda f: None if f is None else np.fromfile(os.path.join(HERE, f), dtype=np.float32).reshape(n, n, n)
        p = oracle.RunParams(**params)
        r = oracle.ref_run(p, load(fd), load(fx))
        out = dict(params=params, dens_file=fd, xhii_file=fx, source="oracle/_ref (unmodified reference)",
                   k=r.k.tolist(), theta=[None if np.isnan(t) else t for t in r.theta],
                   B=r.B.tolist(), npoly=r.npoly.tolist(), kpoly=r.kpoly.tolist(),
                   kmin=r.kmin.tolist(), kmax=r.kmax.tolist())
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(out, f, indent=1)
        print(name, len(r.k))


if __name__ == "__main__":
    main()
