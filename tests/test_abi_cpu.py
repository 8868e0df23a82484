"""C-ABI checks that need no GPU: the library loads, exports every entry
point include/ps_gpu.h declares, rejects bad arguments before touching the
device, and generates the reference's configuration lists."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ps():
    import polyspectrum_b200 as ps
    from polyspectrum_b200 import build
    build.build(quiet=True)
    ps.lib()
    return ps


def declared_symbols():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(ps_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("ps_gpu_init", "ps_gpu_polyspectrum", "ps_gpu_polyspectrum_batch", "ps_gpu_grad",
                 "ps_gpu_finalize", "ps_gpu_strerror", "ps_make_configs"):
        assert must in names


def test_library_exports_every_declared_symbol(ps):
    lib = ps.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_has_no_torch_dependency():
    import subprocess
    out = subprocess.run(["ldd", os.path.join(ROOT, "polyspectrum_b200", "libpsgpu.so")],
                         capture_output=True, text=True).stdout
    assert "torch" not in out and "libc10" not in out


def test_strerror_and_bad_arguments(ps):
    lib = ps.lib()
    assert lib.ps_gpu_strerror(0) == b"ok"
    assert lib.ps_gpu_strerror(-8) == b"undefined in the reference"
    h = C.c_void_p()
    assert lib.ps_gpu_create(C.byref(h), 100, 100.0, 1, -1) == -7  # not a supported size
    assert b"supported are" in lib.ps_gpu_last_error()
    assert lib.ps_gpu_create(C.byref(h), 72, 100.0, 1, -1) == -7
    assert lib.ps_gpu_create(C.byref(h), 64, -1.0, 1, -1) == -1
    assert lib.ps_gpu_create(C.byref(h), 64, 100.0, 0, -1) == -1
    assert lib.ps_gpu_create(None, 64, 100.0, 1, -1) == -1
    assert lib.ps_gpu_polyspectrum_batch(None, 1, 0, None, None, None, None) == -1


@pytest.mark.parametrize("n,eq", [(1, 0), (4, 0)])
def test_make_configs_refuses_like_kvectors(ps, n, eq):
    with pytest.raises(ps.PsError):
        ps.read_params_to_kvectors(64, 100.0, n, equilateral=eq, k1=0.3, k2=0.4, num_values=3)


CFG_CASES = [
    dict(n=2, num_values=2, kbinning=0),
    dict(n=2, num_values=1, k1=0.3, kbinning=2),
    dict(n=2, num_values=5, kbinning=3),
    dict(n=3, equilateral=1, num_values=7, kbinning=0),
    dict(n=3, equilateral=1, num_values=7, kbinning=2, dcos_theta=0.1),
    dict(n=3, equilateral=0, k1=0.2, k2=0.5, num_values=16, kbinning=2, dcos_theta=0.1),
    dict(n=3, equilateral=0, k1=0.2, k2=0.5, num_values=16, kbinning=3, dcos_theta=0.3),
    dict(n=3, equilateral=0, k1=0.4, k2=0.4, num_values=1, theta=0.7, kbinning=2, dcos_theta=0.05),
    dict(n=3, equilateral=0, k1=0.2, k2=0.5, num_values=16, kbinning=1),
]


@pytest.mark.parametrize("case", CFG_CASES)
def test_make_configs_matches_oracle_run(ps, ora, case):
    """ps_make_configs gives the arrays the reference's run loop passes to
    polyspectrum() (compared with the oracle's run, which is bit-identical to
    the reference's; DERIVED ranges are outputs and compared elsewhere)."""
    grid, box = 16, 100.0
    p = dict(equilateral=0, k1=0.0, k2=0.0, theta=0.0, kbinwidth=1.0, dcos_theta=0.2)
    p.update(case)
    cfgs, k, th = ps.read_params_to_kvectors(grid, box, p["n"], equilateral=p["equilateral"],
                                             k1=p["k1"], k2=p["k2"], num_values=p["num_values"],
                                             theta=p["theta"], kbinwidth=p["kbinwidth"],
                                             kbinningCase=p["kbinning"], dcosTheta=p["dcos_theta"])
    rp = ora.RunParams(grid_size=grid, box_size=box, which_field=0, **p)
    d = np.random.default_rng(0).standard_normal((grid,) * 3).astype(np.float32)
    r = ora.ora_run(rp, d)
    np.testing.assert_array_equal(k, r.k)
    n = p["n"]
    kp = np.array([[cfgs[i].k[j] for j in range(n)] for i in range(len(k))])
    np.testing.assert_array_equal(kp, r.kpoly)
    if p["kbinning"] != 1:
        lo = np.array([[cfgs[i].kmin[j] for j in range(n)] for i in range(len(k))])
        hi = np.array([[cfgs[i].kmax[j] for j in range(n)] for i in range(len(k))])
        np.testing.assert_array_equal(lo, r.kmin)
        np.testing.assert_array_equal(hi, r.kmax)
    if n == 3 and p["equilateral"] != 1 and p["num_values"] > 1:
        np.testing.assert_array_equal(th, r.theta)


def test_fault_spec_parsing(ps):
    """ps_gpu_debug_fault arms the host-side injector without touching a GPU;
    malformed specs are refused."""
    lib = ps.lib()
    for good in (b"alloc:1", b"read:3", b"launch:2", b"wait:1", b"alloc:5,read:1", b""):
        assert lib.ps_gpu_debug_fault(good) == 0, good
    for bad in (b"alloc", b"alloc:0", b"alloc:-2", b"disk:1", b"alloc:x", b"alloc:1,", b"launch:1x"):
        assert lib.ps_gpu_debug_fault(bad) == -1, bad
        assert b"fault spec" in lib.ps_gpu_last_error()
    assert lib.ps_gpu_debug_fault(None) == 0
