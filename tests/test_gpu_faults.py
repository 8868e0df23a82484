"""Failure paths, exercised by host-side fault injection (ps_gpu_debug_fault;
no GPU fault is ever caused).  The reference exit()s where an allocation or a
read fails (grid.c:24,133, utils.c:96); here each entry point returns the
status of the failure - PS_ERR_OOM for the Nth device or page-locked
allocation, PS_ERR_IO for the Nth input-file read, PS_ERR_CUDA for the Nth
post-launch status check - the context stays destroyable, and once it is
destroyed the device holds exactly the memory it held before it was created.

Each scenario is run once without injection (to load the library's device
code), then with the fault armed at N = 1, 2, ... until an injected run
completes without reaching the Nth event: every allocation site (or read, or
launch check) the scenario passes through fails once."""
import os
import tempfile

import numpy as np
import pytest

from polyspectrum_b200 import synth

pytestmark = pytest.mark.gpu

N, BOX = 32, 120.0
CODES = {"alloc": -2, "read": -3, "launch": -4}


def _scenario(ps, paths):
    """Every entry point family on one context, then an FP32-only context
    with host composition; returns the first failing status (0 if none)."""
    import torch

    dens = synth.lognormal_density(N, 2.0, 3)
    xhii = synth.ionised_spheres(N, BOX, 20, 4, median_radius=8.0)
    ctx = None
    try:
        ctx = ps.Context(N, BOX)  # both methods
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, (1.0 + dens).astype(np.float32), xhii, use_only_phase=0)
        cfgs, _, _ = ps.read_params_to_kvectors(N, BOX, 3, k1=0.15, k2=0.22, num_values=4,
                                                kbinningCase=ps.PS_BIN_DERIVED)
        ctx.batch(cfgs, ps.PS_FP32_BATCHED, kappa=True)
        ctx.batch(cfgs, ps.PS_FP64_PLAIN)
        p2, _, _ = ps.read_params_to_kvectors(N, BOX, 2, num_values=2)
        ctx.batch(p2, ps.PS_FP32_BATCHED)
        plan = ctx.plan(cfgs, graph=True)
        try:
            plan.execute()
            ctx.set_field_async(ps.PS_FIELD_DENS, torch.from_numpy(dens).cuda())
            plan.submit()
            ctx.synchronize()
        finally:
            plan.close()
        g = cfgs[0]
        ctx.grad(3, [g.k[i] for i in range(3)], [0.0] * 3, [0.0] * 3, 1.0, ps.PS_BIN_DEFAULT)
        ctx.set_field_files(ps.PS_FIELD_XHI_DENS, paths[0], False, paths[1], False)
        ctx.close()
        # an FP32-only context composes host XHI_DENS inputs on host threads
        ctx = ps.Context(N, BOX, methods=ps.PS_FP32_BATCHED)
        pd = torch.from_numpy((1.0 + dens).astype(np.float32)).pin_memory()
        px = torch.from_numpy(xhii).pin_memory()
        ctx.set_field_async(ps.PS_FIELD_XHI_DENS, pd, px)
        ctx.synchronize()
        ctx.batch(cfgs, ps.PS_FP32_BATCHED)
        return 0
    except ps.PsError as e:
        return e.status
    finally:
        if ctx is not None:
            ctx.close()


@pytest.mark.parametrize("kind", ["alloc", "read", "launch"])
def test_injected_failures_return_status_and_leak_nothing(gpu_lib, kind):
    import torch

    ps = gpu_lib
    with tempfile.TemporaryDirectory() as td:
        paths = [os.path.join(td, "dens.raw"), os.path.join(td, "xhii.raw")]
        (1.0 + synth.lognormal_density(N, 2.0, 5)).astype(np.float32).tofile(paths[0])
        synth.ionised_spheres(N, BOX, 20, 6, median_radius=8.0).tofile(paths[1])
        ps.debug_fault(None)
        assert _scenario(ps, paths) == 0
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        hits = 0
        for n in range(1, 400):
            ps.debug_fault(f"{kind}:{n}")
            rc = _scenario(ps, paths)
            ps.debug_fault(None)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0, (kind, n, rc)
            if rc == 0:
                break  # the scenario has fewer than n such events
            assert rc == CODES[kind], (kind, n, rc)
            hits += 1
        else:
            pytest.fail(f"{kind}: the scenario kept failing")
        assert hits >= 1
        # the device still works after all of that
        assert _scenario(ps, paths) == 0


def test_bounded_wait_times_out_and_context_recovers(gpu_lib):
    """The r2c pass of the field waits on an mbarrier for the bulk copies of
    its input tile, for at most 0.2 s.  With "wait:1" armed, the barrier
    expects 16 bytes more than the copies bring (they still complete), so the
    wait runs out: the load returns PS_ERR_TIMEOUT, and the next load on the
    same context gives the results of a normal one."""
    import torch

    ps = gpu_lib
    dens = torch.from_numpy(synth.lognormal_density(N, 2.0, 7)).cuda()
    cfgs, _, _ = ps.read_params_to_kvectors(N, BOX, 3, k1=0.15, k2=0.22, num_values=4, kbinningCase=ps.PS_BIN_DEFAULT)
    with ps.Context(N, BOX, methods=ps.PS_FP32_BATCHED) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_DENS, dens)
        B0, N0, _, _ = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
        ps.debug_fault("wait:1")
        try:
            with pytest.raises(ps.PsError) as err:
                ctx.get_FT_field(ps.PS_FIELD_DENS, dens)
            assert err.value.status == -5, err.value
        finally:
            ps.debug_fault(None)
        ctx.get_FT_field(ps.PS_FIELD_DENS, dens)
        B1, N1, _, _ = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
    np.testing.assert_array_equal(B1, B0)
    np.testing.assert_array_equal(N1, N0)
