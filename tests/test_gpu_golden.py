"""GPU results against the committed golden fixtures produced by the
unmodified reference (tests/golden/make_golden.py).  Same tolerances as
test_gpu_parity.py."""
import glob
import json
import os

import numpy as np
import pytest

from oracle import RunResult
from test_gpu_parity import check

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(path):
    with open(path) as f:
        g = json.load(f)
    n = g["params"]["grid_size"]
    raw = lambda f: None if f is None else np.fromfile(os.path.join(GOLDEN, f), dtype=np.float32).reshape(n, n, n)
    return g, raw(g["dens_file"]), raw(g["xhii_file"])


@pytest.mark.parametrize("method", [1, 2], ids=["plain64", "batched32"])
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.json"))),
                         ids=lambda p: os.path.basename(p)[:-5])
def test_golden(gpu_lib, path, method):
    ps = gpu_lib
    g, dens, xhii = load(path)
    p = g["params"]
    n = p["grid_size"]
    with ps.Context(n, p["box_size"]) as ctx:
        ctx.get_FT_field(p["which_field"], dens, xhii, use_only_phase=p.get("use_only_phase", 0))
        got = ps.run_sweep(ctx, n, p["box_size"], p["n"], method=method,
                           equilateral=p.get("equilateral", 0), k1=p.get("k1", 0.0),
                           k2=p.get("k2", 0.0), num_values=p["num_values"],
                           theta=p.get("theta", 0.0), kbinwidth=p["kbinwidth"],
                           kbinningCase=p["kbinning"], dcosTheta=p["dcos_theta"])
    ref = RunResult(np.array(g["k"]), np.array([np.nan if t is None else t for t in g["theta"]]),
                    np.array(g["B"]), np.array(g["npoly"]), np.array(g["kpoly"]),
                    np.array(g["kmin"]), np.array(g["kmax"]))
    check(ref, got, method, os.path.basename(path))
    if p["kbinning"] == 1:
        np.testing.assert_array_equal(got.kmin, ref.kmin)
        np.testing.assert_array_equal(got.kmax, ref.kmax)
