"""ps_gpu_power_spectrum_noalloc: the power spectrum entry point for callers
that may not allocate device memory (for example code running while a CUDA
stream is captured into a graph, where cudaMalloc is not allowed, or hosts
whose GPU memory belongs to another allocator).  Its working memory is a
fixed device array inside the library instead of cudaMalloc'd buffers.

Checked through the C-ABI against the context-based entry point
(ps_gpu_polyspectrum_batch, PS_FP32_BATCHED) on the same field and shells, on
two calls in a row (the second reuses the scratch the first left behind),
with the batched-method tolerance of the other parity tests: |dP| <= 1e-5 |P|
and exact polygon counts.  This file is collected last."""
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


@pytest.mark.parametrize("n_grid,phase", [(32, 0), (64, 1), (16, 0)])
def test_noalloc_matches_context_entry_point(n_grid, phase):
    import torch

    import polyspectrum_b200 as ps
    from polyspectrum_b200 import synth

    lib = ps.lib()
    fn = _noalloc(lib)
    box = 150.0
    L = float(np.float32(box))
    field = synth.lognormal_density(n_grid, 2.0, 21)
    dev = torch.from_numpy(field).cuda()
    cfgs, k, _ = ps.read_params_to_kvectors(n_grid, box, 2, num_values=2)
    with ps.Context(n_grid, box, methods=ps.PS_FP32_BATCHED) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_DENS, dev, use_only_phase=phase)
        B_ref, N_ref, _, _ = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
    ks = np.ascontiguousarray(k, dtype=np.float64)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    for call in range(2):
        P = np.zeros(len(ks))
        Np = np.zeros(len(ks))
        rc = fn(n_grid, L, C.c_void_p(dev.data_ptr()), phase, len(ks), dp(ks), 1.0, dp(P), dp(Np),
                None)
        assert rc == 0, lib.ps_gpu_last_error()
        np.testing.assert_array_equal(Np, N_ref, err_msg=f"call {call}")
        assert np.all(np.abs(P - B_ref) <= 1e-5 * np.abs(B_ref)), (call, P, B_ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    import polyspectrum_b200 as ps

    lib = ps.lib()
    fn = _noalloc(lib)
    dev = torch.zeros(8, device="cuda")
    ks = np.array([0.1, 0.2])
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    out = np.zeros(2)
    assert fn(128, 100.0, C.c_void_p(dev.data_ptr()), 0, 2, dp(ks), 1.0, dp(out), dp(out), None) == -1
    assert b"64" in lib.ps_gpu_last_error()
    assert fn(32, 100.0, C.c_void_p(dev.data_ptr()), 0, 0, dp(ks), 1.0, dp(out), dp(out), None) == -1
