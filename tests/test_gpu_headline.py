"""The benchmark workload checked against the oracle at its own size.

Workload: XHI_DENS = dens*(1 - xHII) on a 512^3 grid in a 400 Mpc/h box
(xHII from 32000 seeded ionised spheres, dens = 1 + lognormal delta with
P ~ k^-2), phase-only, DERIVED binning, kbinwidth 1; four (k1, k2) theta
sweeps {(0.2,0.5), (0.5,0.8), (0.8,1.2), (1.0,1.5)} h/Mpc of 16 bins each =
64 bispectrum configurations, evaluated by the batched FP32 method in one
call.  Its four pair groups run on 128-, 192-, 320- and 384-point sub-grids.

The oracle (the reference's algorithm restated in C, bit-identical to the
unmodified reference, FP64 throughout) evaluates one configuration of each of
the groups on 192-, 320- and 384-point sub-grids at 512^3 (about half a minute
each on the host cores); bench.py checks a configuration of the fourth group
against the unmodified reference itself in its cpu-baseline leg.  Tolerance:
|dB| <= 1e-5 |B| with no absolute floor, polygon counts exact, DERIVED
k-ranges bit-identical.  The same 64 configurations loaded from device arrays
(the composition then runs in the r2c loader instead of on host threads) give
bit-identical results, and counting polygons with FP64 transforms of the unit
shells instead of the exact enumeration gives the same counts and B."""
import numpy as np
import pytest

from polyspectrum_b200 import synth

pytestmark = pytest.mark.gpu

N, BOX = 512, 400.0
PAIRS = [(0.2, 0.5), (0.5, 0.8), (0.8, 1.2), (1.0, 1.5)]
CHECKED = [(1, 5), (2, 8), (3, 12)]  # (pair index, theta index)


def test_headline_sweep_matches_oracle(gpu_lib, ora):
    import ctypes as C

    import torch

    ps = gpu_lib
    dens, xhii = synth.xhi_dens_inputs(N, BOX, 32000, 3, 2.0, 4)
    allc = []
    for k1, k2 in PAIRS:
        cfgs, _, _ = ps.read_params_to_kvectors(N, BOX, 3, k1=k1, k2=k2, num_values=16,
                                                kbinningCase=ps.PS_BIN_DERIVED)
        allc += [cfgs[i] for i in range(len(cfgs))]
    arr = (ps.ps_cfg * len(allc))()
    for i, g in enumerate(allc):
        C.memmove(C.byref(arr[i]), C.byref(g), C.sizeof(ps.ps_cfg))
    with ps.Context(N, BOX, methods=ps.PS_FP32_BATCHED) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        B, Np, kap, out = ctx.batch(arr, ps.PS_FP32_BATCHED, kappa=True)
        kmin = np.array([[out[q].kmin[j] for j in range(3)] for q in range(64)])
        kmax = np.array([[out[q].kmax[j] for j in range(3)] for q in range(64)])
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, torch.from_numpy(dens).cuda(), torch.from_numpy(xhii).cuda(),
                         use_only_phase=1)
        Bd, Npd, _, _ = ctx.batch(arr, ps.PS_FP32_BATCHED)
        # the counts of the FP64 unit-shell transforms (the reference's dataflow)
        plan = ctx.plan(arr, graph=False, fft_counts=True)
        Bf, Npf, _, _ = plan.execute()
        plan.close()
    np.testing.assert_array_equal(Bd, B)
    np.testing.assert_array_equal(Npd, Np)
    np.testing.assert_array_equal(Npf, Np)
    np.testing.assert_array_equal(Bf, B)
    assert np.all(np.isfinite(B)) and np.all(Np > 0)
    assert np.all(np.isfinite(kap)) and np.all(kap >= 1.0)
    for pi, ti in CHECKED:
        k1, k2 = PAIRS[pi]
        p = ora.RunParams(grid_size=N, box_size=BOX, which_field=2, use_only_phase=1, n=3, equilateral=0,
                          k1=k1, k2=k2, num_values=16, kbinwidth=1.0, kbinning=1)
        ref = ora.ora_run(p, dens, xhii, max_cfg=1, first=ti)
        q = 16 * pi + ti
        rel = abs(B[q] - ref.B[0]) / abs(ref.B[0])
        assert rel <= 1e-5, (pi, ti, B[q], ref.B[0], rel, kap[q])
        assert Np[q] == np.rint(ref.npoly[0]), (pi, ti, Np[q], ref.npoly[0])
        np.testing.assert_array_equal(kmin[q], ref.kmin[0])
        np.testing.assert_array_equal(kmax[q], ref.kmax[0])
