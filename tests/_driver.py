"""Run directories for the command-line driver (polyspectrum_b200/ps_run) and
the reference executable (oracle/_ref/polyspectrum): an ini file with the
reference's keys, raw input grids, an output directory."""
from __future__ import annotations

import os
import subprocess

import numpy as np

from _cases import fields

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PS_RUN = os.path.join(ROOT, "polyspectrum_b200", "ps_run")
BINNING = {0: "DEFAULT", 1: "DERIVED_BINNING", 2: "GIVEN_BINNING", 3: "WATKINSON"}
FIELD = {0: "DENS", 1: "XHII", 2: "XHI_DENS"}


def make_run(tmp, n_grid=16, box=100.0, which=2, gas_dp=0, ion_dp=1, n=3, equilateral=0, k1=0.2, k2=0.3,
             num_values=4, theta=0.5, kbinwidth=1.0, kbinning=0, dcos=0.1, phase=0, write_np=1,
             out_dir="out", extra_lines=(), drop_keys=()):
    """Write inputs and an ini file under tmp; returns the ini path."""
    os.makedirs(os.path.join(tmp, "out"), exist_ok=True)
    dens, xhii = fields(n_grid, box)
    dens = (1.0 + dens.astype(np.float64))
    (dens if gas_dp == 1 else dens.astype(np.float32)).tofile(os.path.join(tmp, "dens.raw"))
    (xhii.astype(np.float64) if ion_dp == 1 else xhii.astype(np.float32)).tofile(os.path.join(tmp, "xhii.raw"))
    keys = [
        ("Grid", [("gridsize", n_grid), ("boxsize", f"{box!r}    # in h^-1 cMpc"),
                  ("gasInputsInDoublePrecision", gas_dp), ("ionInputsInDoublePrecision", ion_dp),
                  ("densityFile", "dens.raw"), ("ionFile", "xhii.raw")]),
        ("Cosmology", [("hubble_h", 0.7), ("omega_b", 0.0456), ("omega_m", 0.27), ("omega_l", 0.73),
                       ("sigma8", 0.8), ("Y", 0.25)]),
        ("Polyspectrum", [("whichField", FIELD[which] if isinstance(which, int) else which),
                          ("useOnlyPhase", phase), ("n", n), ("equilateral", equilateral), ("k1", repr(k1)),
                          ("k2", repr(k2)), ("numValues", num_values), ("theta", repr(theta)),
                          ("kbinwidth", repr(kbinwidth)), ("kbinningCase", BINNING[kbinning]),
                          ("cosThetaBinwidth", repr(dcos))]),
        ("Output", [("output_dir", out_dir), ("output_basename", "run"), ("write_numpolygons", write_np)]),
    ]
    lines = ["# written by tests/_driver.py"]
    for sec, kv in keys:
        lines += ["", f"[{sec}]"]
        lines += [f"{k} = {v}" for k, v in kv if k not in drop_keys]
    lines += list(extra_lines)
    path = os.path.join(tmp, "run.ini")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def run_driver(ini, *args, cwd=None, timeout=600.0):
    return subprocess.run([PS_RUN, *args, ini], cwd=cwd, capture_output=True, text=True, timeout=timeout)


def output_file(stdout: str) -> str:
    for line in stdout.splitlines():
        if line.startswith("FILENAME : "):
            return line[len("FILENAME : "):]
    raise AssertionError("no FILENAME line in:\n" + stdout)


def dry_run_configs(stdout: str):
    """(theta, k) per configuration from `ps_run --dry-run`."""
    out = []
    for line in stdout.splitlines():
        if line.startswith("config "):
            f = dict(t.split("=", 1) for t in line.split() if "=" in t)
            out.append((float(f["theta"]), float(f["k"])))
    return out
