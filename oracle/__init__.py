"""ctypes bindings of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the cpu-baseline / reference legs of
bench.py import this package, and only as the checker.  Two libraries:

* ``_build/libps_oracle.so`` - this repository's C restatement (ps_oracle.c);
  builds from committed sources anywhere gcc is present.
* ``_ref/libpsref.so`` - the unmodified reference sources compiled against the
  FFT shim by ``make -C oracle ref`` (needs the reference checkout at build
  time; the built library is not committed but travels with the tree).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import math
import os
import subprocess
import sys
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libps_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpsref.so")
REF_EXE = os.path.join(HERE, "_ref", "polyspectrum")  # the reference's own executable (main.c)

FIELD_NAMES = {0: "DENS", 1: "XHII", 2: "XHI_DENS"}
BINNING_NAMES = {0: "DEFAULT", 1: "DERIVED_BINNING", 2: "GIVEN_BINNING", 3: "WATKINSON"}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


# Where the build container keeps the read-only reference checkout; the GPU
# hosts have none (they run the prebuilt oracle/_ref).  $PS_REFERENCE_DIR
# overrides it.
_DEFAULT_REFERENCE = "/root/reference"


def reference_checkout() -> str | None:
    """The reference checkout the Makefile's `ref` target compiles
    ($PS_REFERENCE_DIR, else the build container's checkout), if present."""
    path = os.environ.get("PS_REFERENCE_DIR") or _DEFAULT_REFERENCE
    return path if os.path.isdir(os.path.join(path, "src")) else None


def build_oracle(ref: bool = False) -> None:
    """Build the restatement (and, when asked and the reference checkout is
    present, the reference harness)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref:
        src = reference_checkout()
        if src is None:
            raise FileNotFoundError("reference checkout not present")
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={src}"], check=True)


class _OraParams(C.Structure):
    _fields_ = [
        ("grid_size", C.c_int), ("box_size", C.c_double), ("which_field", C.c_int),
        ("use_only_phase", C.c_int), ("n", C.c_int), ("equilateral", C.c_int),
        ("k1", C.c_double), ("k2", C.c_double), ("num_values", C.c_int),
        ("theta", C.c_double), ("kbinwidth", C.c_double), ("kbinning", C.c_int),
        ("dcos_theta", C.c_double), ("write_numpolygons", C.c_int),
    ]


@dataclass
class RunParams:
    """The confObj keys that shape a run (confObj.c:39-105)."""
    grid_size: int
    box_size: float
    which_field: int = 0          # 0 DENS, 1 XHII, 2 XHI_DENS
    use_only_phase: int = 0
    n: int = 3
    equilateral: int = 0
    k1: float = 0.5
    k2: float = 0.5
    num_values: int = 1
    theta: float = 0.5
    kbinwidth: float = 1.0
    kbinning: int = 0             # 0 DEFAULT, 1 DERIVED, 2 GIVEN, 3 WATKINSON
    dcos_theta: float = 0.1
    write_numpolygons: int = 1

    def to_c(self) -> _OraParams:
        return _OraParams(self.grid_size, self.box_size, self.which_field, self.use_only_phase,
                          self.n, self.equilateral, self.k1, self.k2, self.num_values, self.theta,
                          self.kbinwidth, self.kbinning, self.dcos_theta, self.write_numpolygons)


@dataclass
class RunResult:
    k: np.ndarray
    theta: np.ndarray
    B: np.ndarray
    npoly: np.ndarray
    kpoly: np.ndarray
    kmin: np.ndarray
    kmax: np.ndarray
    t_forward: float = math.nan
    t_configs: float = math.nan
    extra: dict = field(default_factory=dict)


@contextlib.contextmanager
def c_stdout_to_stderr():
    """Send what C code prints on stdout (the reference's progress printf's,
    e.g. polyspectrum.c:142, input_field.c:46) to stderr while the block runs,
    so a caller's stdout carries only its own output."""
    libc = C.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return C.CDLL(path)


_ora = None


def oracle_lib() -> C.CDLL:
    global _ora
    if _ora is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle(ref=False)
        lib = _load(ORACLE_SO)
        lib.ora_filter.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, _u8]
        lib.ora_filter.restype = None
        lib.ora_filter_derived.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _u8,
                                           C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.ora_filter_derived.restype = None
        lib.ora_forward.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                    _dp]
        lib.ora_forward.restype = C.c_int
        lib.ora_polyspectrum.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp, C.c_double,
                                         C.c_int, C.c_double, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
        lib.ora_polyspectrum.restype = C.c_double
        lib.ora_num_polygons.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, C.c_int,
                                         C.c_double]
        lib.ora_num_polygons.restype = C.c_double
        lib.ora_num_configs.argtypes = [C.POINTER(_OraParams)]
        lib.ora_num_configs.restype = C.c_int
        lib.ora_run.argtypes = [C.POINTER(_OraParams), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.ora_run.restype = C.c_int
        _ora = lib
    return _ora


def _fields_arg(which: int, dens, xhii):
    is_double = None
    ptrs = []
    keep = []
    for a in (dens, xhii):
        if a is None:
            ptrs.append(None)
            continue
        a = np.ascontiguousarray(a)
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float32)
        d = 1 if a.dtype == np.float64 else 0
        if is_double is None:
            is_double = d
        elif is_double != d:
            raise ValueError("dens and xhii must share a dtype")
        keep.append(a)
        ptrs.append(a.ctypes.data_as(C.c_void_p))
    return ptrs, (is_double or 0), keep


def ora_forward(n: int, which: int, dens, xhii=None, use_only_phase: int = 0) -> np.ndarray:
    """Full complex spectrum (N,N,N) complex128 exactly as get_FT_field + phase."""
    (pd, px), is_double, keep = _fields_arg(which, dens, xhii)
    out = np.empty(2 * n ** 3, dtype=np.float64)
    oracle_lib().ora_forward(n, which, pd, px, is_double, use_only_phase, out)
    del keep
    return out.view(np.complex128).reshape(n, n, n)


def ora_filter(n, kind, k=0.0, kmin=0.0, kmax=0.0, binwidth=1.0, boxsize=1.0) -> np.ndarray:
    out = np.empty(n ** 3, dtype=np.uint8)
    oracle_lib().ora_filter(n, kind, k, kmin, kmax, binwidth, boxsize, out)
    return out.reshape(n, n, n)


def ora_filter_derived(n, k, binwidth, boxsize):
    out = np.empty(n ** 3, dtype=np.uint8)
    lo, hi = C.c_double(), C.c_double()
    oracle_lib().ora_filter_derived(n, k, binwidth, boxsize, out, C.byref(lo), C.byref(hi))
    return out.reshape(n, n, n), lo.value, hi.value


def ora_polyspectrum(n, dk, legs_k, kmin, kmax, binwidth, binning, boxsize):
    """Returns (B, sumD, sumI, kmin_after, kmax_after)."""
    dk = np.ascontiguousarray(dk, dtype=np.complex128).view(np.float64).reshape(-1)
    k = np.ascontiguousarray(legs_k, dtype=np.float64)
    lo = np.array(kmin, dtype=np.float64)
    hi = np.array(kmax, dtype=np.float64)
    sd, si = C.c_double(), C.c_double()
    b = oracle_lib().ora_polyspectrum(n, dk, len(k), k, lo, hi, binwidth, binning, boxsize,
                                      C.byref(sd), C.byref(si))
    return b, sd.value, si.value, lo, hi


def ora_num_polygons(n, legs_k, kmin, kmax, binwidth, binning, boxsize):
    k = np.ascontiguousarray(legs_k, dtype=np.float64)
    lo = np.array(kmin, dtype=np.float64)
    hi = np.array(kmax, dtype=np.float64)
    return oracle_lib().ora_num_polygons(n, len(k), k, lo, hi, binwidth, binning, boxsize)


def ora_run(p: RunParams, dens, xhii=None, max_cfg: int | None = None, first: int = 0) -> RunResult:
    """Configurations [first, first + max_cfg) of the run (all from `first`
    when max_cfg is None), as the reference's run loop computes them."""
    lib = oracle_lib()
    cp = p.to_c()
    ncfg = lib.ora_num_configs(C.byref(cp))
    if ncfg < 0:
        raise ValueError("configuration refused by the reference's kvectors (n>3 or n<2)")
    ncfg = max(0, ncfg - first)
    if max_cfg is not None:
        ncfg = min(ncfg, max_cfg)
    which = p.which_field
    (pd, px), is_double, keep = _fields_arg(which, dens, xhii)
    out = [np.zeros(ncfg) for _ in range(4)] + [np.zeros(ncfg * p.n) for _ in range(3)]
    got = lib.ora_run(C.byref(cp), pd, px, is_double, first, ncfg, *out)
    del keep
    if got < 0:
        raise RuntimeError("ora_run failed")
    k, th, b, npol, kp, kl, kh = out
    return RunResult(k, th, b, npol, kp.reshape(ncfg, p.n), kl.reshape(ncfg, p.n),
                     kh.reshape(ncfg, p.n))


# ---------------------------------------------------------------- reference
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_exe_available() -> bool:
    return os.path.exists(REF_EXE)


def run_ref_exe(ini_path: str, cwd: str | None = None, timeout: float = 600.0) -> subprocess.CompletedProcess:
    """Run the reference executable on an ini file (serial build, shim FFT)."""
    return subprocess.run([REF_EXE, ini_path], cwd=cwd, capture_output=True, text=True, timeout=timeout)


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = _load(REF_SO)
        lib.ref_num_configs_ini.argtypes = [C.c_char_p]
        lib.ref_num_configs_ini.restype = C.c_int
        lib.ref_run_ini.argtypes = [C.c_char_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                                    _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.ref_run_ini.restype = C.c_int
        _ref = lib
    return _ref


def ref_set_threads(n: int) -> None:
    """Threads of the FFT shim inside oracle/_ref (0: $PS_SHIM_THREADS, else
    every CPU)."""
    lib = ref_lib()
    lib.ps_shim_set_threads.argtypes = [C.c_int]
    lib.ps_shim_set_threads.restype = None
    lib.ps_shim_set_threads(int(n))


def ora_set_threads(n: int) -> None:
    """Threads of the FFT shim inside the restatement's library."""
    lib = oracle_lib()
    lib.ps_shim_set_threads.argtypes = [C.c_int]
    lib.ps_shim_set_threads.restype = None
    lib.ps_shim_set_threads(int(n))


def write_ini(path: str, p: RunParams, dens_file: str, ion_file: str, is_double: int,
              out_dir: str) -> None:
    """An iniFile.ini with the reference's keys (iniFile.ini, README.rst:59-104)."""
    txt = f"""[Grid]
gridsize = {p.grid_size}
boxsize = {p.box_size!r}
gasInputsInDoublePrecision = {is_double}
ionInputsInDoublePrecision = {is_double}
densityFile = {dens_file}
ionFile = {ion_file}

[Cosmology]
hubble_h = 0.7
omega_b = 0.0456
omega_m = 0.27
omega_l = 0.73
sigma8 = 0.8
Y = 0.25

[Polyspectrum]
whichField = {FIELD_NAMES[p.which_field]}
useOnlyPhase = {p.use_only_phase}
n = {p.n}
equilateral = {p.equilateral}
k1 = {p.k1!r}
k2 = {p.k2!r}
numValues = {p.num_values}
theta = {p.theta!r}
kbinwidth = {p.kbinwidth!r}
kbinningCase = {BINNING_NAMES[p.kbinning]}
cosThetaBinwidth = {p.dcos_theta!r}

[Output]
output_dir = {out_dir}
output_basename = oracle
write_numpolygons = {p.write_numpolygons}
"""
    with open(path, "w") as f:
        f.write(txt)


def ref_run(p: RunParams, dens, xhii=None, first: int = 0, count: int = -1) -> RunResult:
    """Run the unmodified reference on in-memory fields (written to raw files,
    read back by the reference's own grid.c readers)."""
    lib = ref_lib()
    with tempfile.TemporaryDirectory(prefix="psref_") as td:
        arrs = [a for a in (dens, xhii) if a is not None]
        is_double = 1 if arrs and np.asarray(arrs[0]).dtype == np.float64 else 0
        dt = np.float64 if is_double else np.float32
        dpath = os.path.join(td, "dens.raw")
        ipath = os.path.join(td, "ion.raw")
        zeros = np.zeros((p.grid_size,) * 3, dtype=dt)
        np.ascontiguousarray(dens if dens is not None else zeros, dtype=dt).tofile(dpath)
        np.ascontiguousarray(xhii if xhii is not None else zeros, dtype=dt).tofile(ipath)
        ini = os.path.join(td, "iniFile.ini")
        write_ini(ini, p, dpath, ipath, is_double, td)
        with c_stdout_to_stderr():
            total = lib.ref_num_configs_ini(ini.encode())
        ncfg = total - first if count < 0 else min(count, total - first)
        out = [np.zeros(max(ncfg, 1)) for _ in range(4)] + \
              [np.zeros(max(ncfg, 1) * p.n) for _ in range(3)]
        tf, tc = C.c_double(), C.c_double()
        with c_stdout_to_stderr():
            got = lib.ref_run_ini(ini.encode(), first, ncfg, *out, C.byref(tf), C.byref(tc))
    k, th, b, npol, kp, kl, kh = [o[: got * (p.n if i >= 4 else 1)] for i, o in enumerate(out)]
    return RunResult(k, th, b, npol, kp.reshape(got, p.n), kl.reshape(got, p.n),
                     kh.reshape(got, p.n), tf.value, tc.value)
