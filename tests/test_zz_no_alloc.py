"""ps_gpu_power_spectrum_noalloc: the power spectrum entry point for host
programs that may not allocate device memory, because their GPU memory is owned
by another allocator (a framework's caching pool that has reserved the device,
or a fixed real-time memory budget).  Its working memory is a fixed device
array inside the library instead of cudaMalloc'd buffers.

Checked through the C-ABI against the context-based entry point
(ps_gpu_polyspectrum_batch, PS_FP32_BATCHED) on the same field and shells, on
two calls in a row (the second reuses the scratch the first left behind),
with the batched-method tolerance of the other parity tests: |dP| <= 1e-5 |P|
and exact polygon counts; also that a call leaves the device's free memory
unchanged, and that it refuses what its fixed array cannot hold.  This file is
collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.ps_gpu_power_spectrum_noalloc
    f.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double),
                  C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _context_reference(ps, n_grid, box, dev, phase, ks, bw):
    """P(k) and counts of the shells through the context entry point."""
    cfgs = (ps.ps_cfg * len(ks))()
    for i, k in enumerate(ks):
        C.memmove(C.byref(cfgs[i]), C.byref(ps.make_cfg(2, [k, k], kbinwidth=bw)), C.sizeof(ps.ps_cfg))
    with ps.Context(n_grid, box, methods=ps.PS_FP32_BATCHED) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_DENS, dev, use_only_phase=phase)
        B_ref, N_ref, _, _ = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
    return B_ref, N_ref


@pytest.mark.parametrize("n_grid,phase,nshell,bw", [(32, 0, 16, 1.0), (64, 1, 32, 1.0), (16, 0, 8, 1.0),
                                                    (64, 0, 256, 0.7)])
def test_noalloc_matches_context_entry_point(n_grid, phase, nshell, bw):
    import torch

    import polyspectrum_b200 as ps
    from polyspectrum_b200 import synth

    lib = ps.lib()
    fn = _noalloc(lib)
    box = 150.0
    L = float(np.float32(box))
    kf = 2 * np.pi / L
    field = synth.lognormal_density(n_grid, 2.0, 21)
    dev = torch.from_numpy(field).cuda()
    # shells from the fundamental mode up to just below Nyquist
    ks = np.ascontiguousarray(np.linspace(1.0, n_grid / 2 - 1.0, nshell) * kf, dtype=np.float64)
    B_ref, N_ref = _context_reference(ps, n_grid, box, dev, phase, ks, bw)
    assert np.all(N_ref > 0)
    torch.cuda.synchronize()
    free = []
    for call in range(3):
        P = np.zeros(len(ks))
        Np = np.zeros(len(ks))
        free.append(torch.cuda.mem_get_info()[0])
        rc = fn(n_grid, L, C.c_void_p(dev.data_ptr()), phase, len(ks), _dp(ks), bw, _dp(P), _dp(Np), None)
        assert rc == 0, lib.ps_gpu_last_error()
        np.testing.assert_array_equal(Np, N_ref, err_msg=f"call {call}")
        assert np.all(np.abs(P - B_ref) <= 1e-5 * np.abs(B_ref)), (call, P, B_ref)
    free.append(torch.cuda.mem_get_info()[0])
    # the first call may load the library's device code (with the array);
    # after that a call takes no device memory
    assert free[1] == free[2] == free[3], free


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    import polyspectrum_b200 as ps

    lib = ps.lib()
    fn = _noalloc(lib)
    dev = torch.zeros(8, device="cuda")
    ks = np.array([0.1, 0.2])
    out = np.zeros(2)
    ptr = C.c_void_p(dev.data_ptr())
    assert fn(128, 100.0, ptr, 0, 2, _dp(ks), 1.0, _dp(out), _dp(out), None) == -1
    assert b"64" in lib.ps_gpu_last_error()
    assert fn(32, 100.0, ptr, 0, 0, _dp(ks), 1.0, _dp(out), _dp(out), None) == -1
    assert fn(32, 100.0, ptr, 0, 257, _dp(ks), 1.0, _dp(out), _dp(out), None) == -1
    assert fn(32, float("inf"), ptr, 0, 2, _dp(ks), 1.0, _dp(out), _dp(out), None) == -1
    assert fn(32, 100.0, ptr, 0, 2, _dp(ks), 0.0, _dp(out), _dp(out), None) == -1
    assert fn(32, 100.0, ptr, 0, 2, _dp(ks), float("nan"), _dp(out), _dp(out), None) == -1
    assert fn(32, 100.0, ptr, 2, 2, _dp(ks), 1.0, _dp(out), _dp(out), None) == -1
