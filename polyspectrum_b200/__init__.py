"""B200-native polyspectrum estimator (libpsgpu.so) - Python binding.

The product is the C-ABI in include/ps_gpu.h, implemented by the CUDA
library polyspectrum_b200/libpsgpu.so (built in-tree by
``python -m polyspectrum_b200.build``).  This module is a thin ctypes layer
over it for tests, benchmarks and Python users; it never computes anything
itself and raises if the library is missing.

Names follow the reference (annehutter/polyspectrum):
``polyspectrum`` / ``num_polygons`` (polyspectrum.c:51,163),
``get_FT_field`` (input_field.c:40), ``read_params_to_kvectors``
(kvectors.c:46).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpsgpu.so")

PS_OK = 0
PS_FP64_PLAIN = 1
PS_FP32_BATCHED = 2
PS_FIELD_DENS, PS_FIELD_XHII, PS_FIELD_XHI_DENS = 0, 1, 2
PS_BIN_DEFAULT, PS_BIN_DERIVED, PS_BIN_GIVEN, PS_BIN_WATKINSON = 0, 1, 2, 3
PS_MEM_HOST, PS_MEM_DEVICE = 0, 1
PS_MAX_LEGS = 8
ERRORS = {-1: "PS_ERR_ARG", -2: "PS_ERR_OOM", -3: "PS_ERR_IO", -4: "PS_ERR_CUDA",
          -5: "PS_ERR_TIMEOUT", -6: "PS_ERR_NONFINITE", -7: "PS_ERR_UNSUPPORTED",
          -8: "PS_ERR_UNDEFINED"}


class PsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{ERRORS.get(status, status)}: {message}")
        self.status = status


class ps_cfg(C.Structure):
    _fields_ = [("n", C.c_int), ("kbinningCase", C.c_int), ("kbinwidth", C.c_double),
                ("k", C.c_double * PS_MAX_LEGS), ("kmin", C.c_double * PS_MAX_LEGS),
                ("kmax", C.c_double * PS_MAX_LEGS)]


class ps_run_params(C.Structure):
    _fields_ = [("grid_size", C.c_int), ("box_size", C.c_double), ("n", C.c_int),
                ("equilateral", C.c_int), ("k1", C.c_double), ("k2", C.c_double),
                ("num_values", C.c_int), ("theta", C.c_double), ("kbinwidth", C.c_double),
                ("kbinningCase", C.c_int), ("dcosTheta", C.c_double)]


class ps_kernel_stat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_longlong), ("ms", C.c_double),
                ("bytes", C.c_double)]


class ps_load_stats(C.Structure):
    _fields_ = [("rows", C.c_longlong), ("rows_raw", C.c_longlong), ("bytes", C.c_longlong),
                ("compose_s", C.c_double), ("raw_copy_ms", C.c_double), ("next_raw_frac", C.c_double),
                ("host_threads", C.c_int)]


_lib = None


def lib() -> C.CDLL:
    """Load the in-tree CUDA library (fails loudly when it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: build it with `python -m polyspectrum_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
    L.ps_gpu_create.argtypes = [C.POINTER(vp), ip, C.c_double, ip, ip]
    L.ps_gpu_set_field.argtypes = [vp, ip, vp, vp, ip, ip, ip]
    L.ps_gpu_init.argtypes = [C.POINTER(vp), ip, C.c_double, vp, ip, ip, ip]
    L.ps_gpu_polyspectrum.argtypes = [vp, ip, dp, dp, dp, C.c_double, ip, dp, dp]
    L.ps_gpu_polyspectrum_batch.argtypes = [vp, ip, ip, C.POINTER(ps_cfg), dp, dp, dp]
    L.ps_gpu_grad.argtypes = [vp, ip, ip, dp, dp, dp, C.c_double, ip, vp, ip, ip]
    L.ps_make_configs.argtypes = [C.POINTER(ps_run_params), C.POINTER(ps_cfg), ip, dp, dp]
    L.ps_gpu_set_stream.argtypes = [vp, vp]
    L.ps_gpu_last_timing.argtypes = [vp, dp, C.POINTER(C.c_longlong)]
    L.ps_gpu_plan_create.argtypes = [vp, ip, ip, C.POINTER(ps_cfg), ip, C.POINTER(vp)]
    L.ps_gpu_plan_execute.argtypes = [vp, vp, dp, dp, dp, C.POINTER(ps_cfg)]
    L.ps_gpu_plan_destroy.argtypes = [vp]
    L.ps_gpu_plan_destroy.restype = None
    L.ps_gpu_set_field_async.argtypes = [vp, ip, vp, vp, ip, ip, ip]
    L.ps_gpu_set_field_files.argtypes = [vp, ip, C.c_char_p, ip, C.c_char_p, ip, ip]
    L.ps_gpu_load_stats.argtypes = [vp, C.POINTER(ps_load_stats)]
    L.ps_gpu_debug_fault.argtypes = [C.c_char_p]
    L.ps_gpu_plan_results_device.argtypes = [vp, vp, vp]
    L.ps_gpu_upload_bytes.argtypes = [vp]
    L.ps_gpu_upload_bytes.restype = C.c_longlong
    L.ps_gpu_plan_submit.argtypes = [vp, vp, dp, dp, dp, C.POINTER(ps_cfg)]
    L.ps_gpu_synchronize.argtypes = [vp]
    L.ps_gpu_launch_count.argtypes = [vp]
    L.ps_gpu_launch_count.restype = C.c_longlong
    L.ps_gpu_tune_export.argtypes = [vp, C.c_char_p, ip]
    L.ps_gpu_keep_modulus.argtypes = [vp, ip]
    L.ps_gpu_set_spectrum_band.argtypes = [vp, ip]
    L.ps_gpu_plan_launch.argtypes = [vp, vp]
    L.ps_gpu_plan_prepare.argtypes = [vp, vp]
    L.ps_gpu_plan_results.argtypes = [vp, vp, dp, dp, dp, C.POINTER(ps_cfg)]
    L.ps_gpu_plan_band.argtypes = [vp]
    L.ps_gpu_tune_import.argtypes = [vp, C.c_char_p]
    L.ps_gpu_set_profiling.argtypes = [vp, ip]
    L.ps_gpu_kernel_stats.argtypes = [vp, C.POINTER(ps_kernel_stat), ip]
    L.ps_gpu_finalize.argtypes = [vp]
    L.ps_gpu_finalize.restype = None
    L.ps_gpu_strerror.argtypes = [ip]
    L.ps_gpu_strerror.restype = C.c_char_p
    L.ps_gpu_last_error.argtypes = []
    L.ps_gpu_last_error.restype = C.c_char_p
    for name in ("ps_gpu_create", "ps_gpu_set_field", "ps_gpu_init", "ps_gpu_polyspectrum",
                 "ps_gpu_polyspectrum_batch", "ps_gpu_grad", "ps_make_configs",
                 "ps_gpu_set_stream", "ps_gpu_last_timing", "ps_gpu_set_profiling",
                 "ps_gpu_kernel_stats", "ps_gpu_plan_create", "ps_gpu_plan_execute",
                 "ps_gpu_set_field_async", "ps_gpu_plan_submit", "ps_gpu_synchronize",
                 "ps_gpu_tune_export", "ps_gpu_tune_import", "ps_gpu_keep_modulus",
                 "ps_gpu_set_spectrum_band", "ps_gpu_plan_band", "ps_gpu_plan_launch", "ps_gpu_plan_prepare",
                 "ps_gpu_plan_results",
                 "ps_gpu_set_field_files", "ps_gpu_load_stats", "ps_gpu_debug_fault",
                 "ps_gpu_plan_results_device"):
        getattr(L, name).restype = ip
    _lib = L
    return L


def debug_fault(spec: str | None) -> None:
    """Arm host-side fault injection ("alloc:N", "read:N", "launch:N"; None
    disarms): see ps_gpu_debug_fault."""
    _check(lib().ps_gpu_debug_fault(None if spec is None else spec.encode()))


def _check(status: int) -> int:
    if status < 0:
        raise PsError(status, lib().ps_gpu_last_error().decode(errors="replace"))
    return status


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_cfg(n, k, kmin=None, kmax=None, kbinwidth=1.0, kbinningCase=0) -> ps_cfg:
    g = ps_cfg()
    g.n = n
    g.kbinningCase = kbinningCase
    g.kbinwidth = kbinwidth
    for i in range(n):
        g.k[i] = k[i]
        g.kmin[i] = 0.0 if kmin is None else kmin[i]
        g.kmax[i] = 0.0 if kmax is None else kmax[i]
    return g


def read_params_to_kvectors(grid_size, box_size, n, equilateral=0, k1=0.0, k2=0.0, num_values=1,
                            theta=0.0, kbinwidth=1.0, kbinningCase=0, dcosTheta=0.0):
    """Configuration list of a run (kvectors.c:46-147 + run.c:56-84), computed
    by ps_make_configs.  Returns (cfgs, k, theta)."""
    p = ps_run_params(grid_size, box_size, n, equilateral, k1, k2, num_values, theta, kbinwidth,
                      kbinningCase, dcosTheta)
    cnt = _check(lib().ps_make_configs(C.byref(p), None, 0, None, None))
    arr = (ps_cfg * max(cnt, 1))()
    k = np.zeros(max(cnt, 1))
    th = np.zeros(max(cnt, 1))
    _check(lib().ps_make_configs(C.byref(p), arr, cnt, _dptr(k), _dptr(th)))
    return arr, k[:cnt], th[:cnt]


def _field_ptr(a):
    """(pointer, is_double, mem, keepalive) for a numpy array or a torch tensor."""
    if a is None:
        return None, None, None, None
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):  # torch tensor
        import torch
        if a.dtype not in (torch.float32, torch.float64) or not a.is_contiguous():
            raise ValueError("field tensors must be contiguous float32/float64")
        return (C.c_void_p(a.data_ptr()), int(a.dtype == torch.float64),
                PS_MEM_DEVICE if a.is_cuda else PS_MEM_HOST, a)
    arr = np.ascontiguousarray(a)
    if arr.dtype not in (np.float32, np.float64):
        arr = arr.astype(np.float32)
    return arr.ctypes.data_as(C.c_void_p), int(arr.dtype == np.float64), PS_MEM_HOST, arr


class Context:
    """One estimator context (ps_gpu_ctx) on one GPU."""

    def __init__(self, nbins: int, boxsize: float, methods: int = PS_FP64_PLAIN | PS_FP32_BATCHED,
                 device: int = -1, float_box: bool = True):
        self.nbins = nbins
        # grid_t stores the box size as float (grid.h:9)
        self.boxsize = float(np.float32(boxsize)) if float_box else float(boxsize)
        self.methods = methods
        h = C.c_void_p()
        _check(lib().ps_gpu_create(C.byref(h), nbins, self.boxsize, methods, device))
        self._h = h
        self._inflight = []  # arrays an asynchronous call may still read or write

    def close(self):
        if getattr(self, "_h", None):
            lib().ps_gpu_finalize(self._h)
            self._h = None
            self._inflight = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def get_FT_field(self, which: int, dens=None, xhii=None, use_only_phase: int = 0):
        """Load the field(s) and run the forward transform on the device."""
        pd, dd, md, kd = _field_ptr(dens)
        px, dx, mx, kx = _field_ptr(xhii)
        is_double = dd if dd is not None else dx
        mem = md if md is not None else mx
        if dd is not None and dx is not None and (dd != dx or md != mx):
            raise ValueError("dens and xhii must share dtype and memory kind")
        _check(lib().ps_gpu_set_field(self._h, which, pd, px, is_double, mem, use_only_phase))

    set_field = get_FT_field

    def set_field_files(self, which: int, dens_path=None, dens_double: bool = False, xhii_path=None,
                        xhii_double: bool = False, use_only_phase: int = 0):
        """Load the field from raw grid files, streamed to the device in chunks
        (ps_gpu_set_field_files); each file is float or double."""
        enc = lambda p: None if p is None else os.fsencode(p)
        _check(lib().ps_gpu_set_field_files(self._h, which, enc(dens_path), int(bool(dens_double)),
                                            enc(xhii_path), int(bool(xhii_double)), use_only_phase))

    def set_field_async(self, which: int, dens=None, xhii=None, use_only_phase: int = 0):
        """get_FT_field queued behind the work already on the context
        (ps_gpu_set_field_async); the arrays are kept alive until synchronize().
        Host arrays overlap with device work only when page-locked (torch
        tensors from pin_memory())."""
        pd, dd, md, kd = _field_ptr(dens)
        px, dx, mx, kx = _field_ptr(xhii)
        is_double = dd if dd is not None else dx
        mem = md if md is not None else mx
        if dd is not None and dx is not None and (dd != dx or md != mx):
            raise ValueError("dens and xhii must share dtype and memory kind")
        self._inflight.append((kd, kx))
        _check(lib().ps_gpu_set_field_async(self._h, which, pd, px, is_double, mem, use_only_phase))

    def synchronize(self):
        """Wait for all queued work; raises for errors found during submissions."""
        try:
            _check(lib().ps_gpu_synchronize(self._h))
        finally:
            self._inflight = []

    def upload_bytes(self) -> int:
        """Host -> device bytes of the last host field load (ps_gpu_upload_bytes)."""
        return int(lib().ps_gpu_upload_bytes(self._h))

    def load_stats(self) -> dict:
        """Statistics of the last host field load (ps_gpu_load_stats)."""
        st = ps_load_stats()
        _check(lib().ps_gpu_load_stats(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in ps_load_stats._fields_}

    def launch_count(self) -> int:
        """Kernels executed by this context since its creation."""
        return int(lib().ps_gpu_launch_count(self._h))

    def polyspectrum(self, n, k, kmin, kmax, kbinwidth, kbinningCase):
        """polyspectrum() + num_polygons() of one configuration with the
        context's first method.  Returns (B, Npoly, kmin, kmax) (the k ranges
        as written back by DERIVED binning)."""
        k = np.ascontiguousarray(k, dtype=np.float64)
        lo = np.array(kmin, dtype=np.float64)
        hi = np.array(kmax, dtype=np.float64)
        B, Np = C.c_double(), C.c_double()
        _check(lib().ps_gpu_polyspectrum(self._h, n, _dptr(k), _dptr(lo), _dptr(hi), kbinwidth,
                                         kbinningCase, C.byref(B), C.byref(Np)))
        return B.value, Np.value, lo, hi

    def batch(self, cfgs, method: int = PS_FP32_BATCHED, kappa: bool = False):
        """Evaluate a list of ps_cfg.  Returns (B, Npoly, kappa, cfgs-after);
        kappa (condition numbers, one extra pass per sum) only when asked,
        else NaN."""
        if not isinstance(cfgs, C.Array):
            arr = (ps_cfg * len(cfgs))(*cfgs)
        else:
            arr = cfgs
        m = len(arr)
        B = np.zeros(m)
        Np = np.zeros(m)
        kap = np.full(m, np.nan)
        _check(lib().ps_gpu_polyspectrum_batch(self._h, method, m, arr, _dptr(B), _dptr(Np),
                                               _dptr(kap) if kappa else None))
        return B, Np, kap, arr

    def plan(self, cfgs, method: int = PS_FP32_BATCHED, graph: bool = True, kappa: bool = False,
             autotune: bool = False, fft_counts: bool = False):
        """A reusable plan of these configurations (ps_gpu_plan_create)."""
        return Plan(self, cfgs, method, graph, kappa, autotune, fft_counts)

    def set_spectrum_band(self, band: int):
        """Later loads compute only modes with |components| <= band (-1: all)."""
        _check(lib().ps_gpu_set_spectrum_band(self._h, int(band)))

    def keep_modulus(self, on: bool = True):
        """Phase-only loads keep |X| so grad() can differentiate through z/|z|."""
        _check(lib().ps_gpu_keep_modulus(self._h, int(bool(on))))

    def tune_export(self) -> str:
        """The autotuned sub-grid choices of this context (ps_gpu_tune_export)."""
        n = _check(lib().ps_gpu_tune_export(self._h, None, 0))
        buf = C.create_string_buffer(n + 1)
        _check(lib().ps_gpu_tune_export(self._h, buf, n + 1))
        return buf.value.decode()

    def tune_import(self, text: str):
        _check(lib().ps_gpu_tune_import(self._h, text.encode()))

    def grad(self, n, k, kmin, kmax, kbinwidth, kbinningCase, method=PS_FP64_PLAIN,
             out=None, double=True):
        k = np.ascontiguousarray(k, dtype=np.float64)
        lo = np.ascontiguousarray(kmin, dtype=np.float64)
        hi = np.ascontiguousarray(kmax, dtype=np.float64)
        if out is None:
            out = np.zeros((self.nbins,) * 3, dtype=np.float64 if double else np.float32)
        po, do, mo, ko = _field_ptr(out)
        _check(lib().ps_gpu_grad(self._h, method, n, _dptr(k), _dptr(lo), _dptr(hi), kbinwidth,
                                 kbinningCase, po, do, mo))
        return out

    def last_timing(self):
        ms = C.c_double()
        n = C.c_longlong()
        _check(lib().ps_gpu_last_timing(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def set_profiling(self, on: bool):
        _check(lib().ps_gpu_set_profiling(self._h, int(bool(on))))

    def kernel_stats(self) -> list[dict]:
        """Per kernel family: launches, summed device ms, summed algorithmic bytes."""
        buf = (ps_kernel_stat * 64)()
        cnt = min(_check(lib().ps_gpu_kernel_stats(self._h, buf, 64)), 64)
        return [dict(name=buf[i].name.decode(), launches=buf[i].launches, ms=buf[i].ms,
                     bytes=buf[i].bytes) for i in range(cnt)]

    def set_stream(self, stream_ptr: int | None):
        _check(lib().ps_gpu_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))


PS_PLAN_GRAPH = 1
PS_PLAN_KAPPA = 2
PS_PLAN_AUTOTUNE = 4
PS_PLAN_FFT_COUNTS = 8


class Plan:
    """ps_gpu_plan: a batch planned once, executed per field (CUDA graph replay
    with graph=True)."""

    def __init__(self, ctx: Context, cfgs, method=PS_FP32_BATCHED, graph=True, kappa=False, autotune=False,
                 fft_counts=False):
        arr = cfgs if isinstance(cfgs, C.Array) else (ps_cfg * len(cfgs))(*cfgs)
        self.ctx = ctx
        self.n = len(arr)
        self.kappa = kappa
        h = C.c_void_p()
        flags = ((PS_PLAN_GRAPH if graph else 0) | (PS_PLAN_KAPPA if kappa else 0)
                 | (PS_PLAN_AUTOTUNE if autotune else 0) | (PS_PLAN_FFT_COUNTS if fft_counts else 0))
        _check(lib().ps_gpu_plan_create(ctx.handle, method, self.n, arr, flags, C.byref(h)))
        self._h = h

    def execute(self):
        B = np.zeros(self.n)
        Np = np.zeros(self.n)
        kap = np.full(self.n, np.nan)
        out = (ps_cfg * max(self.n, 1))()
        _check(lib().ps_gpu_plan_execute(self.ctx.handle, self._h, _dptr(B), _dptr(Np),
                                         _dptr(kap) if self.kappa else None, out))
        return B, Np, kap, out

    @property
    def band(self) -> int:
        """Largest |component| of a mode this plan reads (ps_gpu_plan_band)."""
        return _check(lib().ps_gpu_plan_band(self._h))

    def launch(self):
        """Queue one execution, results left on the device (ps_gpu_plan_launch)."""
        _check(lib().ps_gpu_plan_launch(self.ctx.handle, self._h))

    def prepare(self):
        """Queue the field-independent parts of the next execution (DERIVED
        k-ranges, exact counts) on the side stream, so that a field load queued
        next overlaps them (ps_gpu_plan_prepare)."""
        _check(lib().ps_gpu_plan_prepare(self.ctx.handle, self._h))

    def results(self):
        """Results of the latest execution (waits): (B, Npoly, kappa, cfgs_out)."""
        B = np.zeros(self.n)
        Np = np.zeros(self.n)
        kap = np.full(self.n, np.nan)
        out = (ps_cfg * max(self.n, 1))()
        _check(lib().ps_gpu_plan_results(self.ctx.handle, self._h, _dptr(B), _dptr(Np),
                                         _dptr(kap) if self.kappa else None, out))
        return B, Np, kap, out

    def results_to_device(self, dst_ptr: int):
        """Queue a copy of the latest execution's results into device memory
        (8 doubles per configuration, ps_gpu_plan_results_device)."""
        _check(lib().ps_gpu_plan_results_device(self.ctx.handle, self._h, C.c_void_p(dst_ptr)))

    def submit(self) -> "Submission":
        """Queue one execution on the field most recently loaded (ps_gpu_plan_submit);
        the returned arrays are filled once ctx.synchronize() returns."""
        sub = Submission(self.n, self.kappa)
        _check(lib().ps_gpu_plan_submit(self.ctx.handle, self._h, _dptr(sub.B), _dptr(sub.npoly),
                                        _dptr(sub.kappa) if self.kappa else None, sub.cfgs))
        self.ctx._inflight.append(sub)
        return sub

    def close(self):
        if getattr(self, "_h", None):
            lib().ps_gpu_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Submission:
    """Output arrays of one asynchronous plan execution."""

    def __init__(self, n: int, kappa: bool):
        self.B = np.zeros(n)
        self.npoly = np.zeros(n)
        self.kappa = np.full(n, np.nan)
        self.cfgs = (ps_cfg * max(n, 1))()


@dataclass
class SweepResult:
    k: np.ndarray
    theta: np.ndarray
    B: np.ndarray
    npoly: np.ndarray
    kmin: np.ndarray
    kmax: np.ndarray
    kappa: np.ndarray


def run_sweep(ctx: Context, grid_size, box_size, n, method=PS_FP32_BATCHED, **params) -> SweepResult:
    """The run.c:56-107 loop for one parameter set on a loaded field."""
    cfgs, k, th = read_params_to_kvectors(grid_size, box_size, n, **params)
    B, Np, kap, arr = ctx.batch(cfgs, method)
    kmin = np.array([[arr[i].kmin[j] for j in range(n)] for i in range(len(arr))])
    kmax = np.array([[arr[i].kmax[j] for j in range(n)] for i in range(len(arr))])
    return SweepResult(k, th, B, Np, kmin, kmax, kap)
