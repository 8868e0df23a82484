"""The named run configurations at their own sizes (synthetic inputs with the
stated shapes, spectra and seeds):

  * 128^3 DENS lognormal (P ~ k^-2, seed 1), L = 200: equilateral sweep of 64
    values and the power spectrum over all shells, FP64 plain against the
    oracle (the reference's algorithm on the CPU), batched against both;
  * 256^3 XHII (4000 spheres, seed 2), L = 300: k1 = 0.5, k2 = 1.0, 20 theta
    bins, GIVEN binning, cosThetaBinwidth 0.1; all 20 bins against the oracle,
    plain FP64 and batched FP32 (1e-5 relative, no absolute floor);
  * 1024^3 DENS lognormal (P ~ k^-1.5, seed 8), L = 1000: power spectrum over
    all 512 shells plus 128 triangle configurations (64 equilateral, 64
    isosceles k1 = k2 = 0.3); batched FP32 against plain FP64 on a sample of
    the triangles and on all shells.  The field is drawn on the GPU (torch)
    with the same recipe as polyspectrum_b200/synth.py, to keep the test's host
    memory and time small.

Tolerances as in test_gpu_parity.py: plain FP64 1e-9 relative to the oracle,
batched 1e-5 relative plus 1e-6 of the sweep's max |B|, counts exact."""
import numpy as np
import pytest

from polyspectrum_b200 import synth

pytestmark = pytest.mark.gpu


def _close(got, ref, rt, at):
    scale = np.nanmax(np.abs(ref))
    ok = np.abs(got - ref) <= rt * np.abs(ref) + at * scale
    return bool(ok.all()), np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)


def test_config_128_equilateral_and_power(gpu_lib, ora):
    ps = gpu_lib
    n, box = 128, 200.0
    dens = synth.lognormal_density(n, 2.0, 1)
    for nleg, eq in ((3, 1), (2, 0)):
        p = ora.RunParams(grid_size=n, box_size=box, which_field=0, use_only_phase=0, n=nleg, equilateral=eq,
                          num_values=64, kbinwidth=1.0, kbinning=0)
        ref = ora.ora_run(p, dens)
        with ps.Context(n, box) as ctx:
            ctx.get_FT_field(ps.PS_FIELD_DENS, dens)
            cfgs, k, _ = ps.read_params_to_kvectors(n, box, nleg, equilateral=eq, num_values=64)
            B64, N64, _, _ = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
            B32, N32, _, _ = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
        has = np.rint(ref.npoly) != 0
        ok, _ = _close(B64[has], ref.B[has], 1e-9, 1e-11)
        assert ok, (nleg, B64, ref.B)
        ok, _ = _close(B32[has], ref.B[has], 1e-5, 1e-6)
        assert ok, (nleg, B32, ref.B)
        np.testing.assert_array_equal(N32, np.rint(ref.npoly))
        assert np.all(np.abs(N64 - ref.npoly) <= 1e-7 * np.maximum(1.0, ref.npoly))


def test_config_256_xhii_given(gpu_lib, ora):
    """All 20 theta bins against the oracle: plain FP64 to 1e-9, batched FP32
    to 1e-5 relative with no absolute floor (each bin's condition number is
    computed too, so a bin near a zero crossing would show why), counts
    exact, the k lists identical."""
    ps = gpu_lib
    n, box = 256, 300.0
    xhii = synth.ionised_spheres(n, box, 4000, 2)
    with ps.Context(n, box) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHII, None, xhii)
        cfgs, k, th = ps.read_params_to_kvectors(n, box, 3, k1=0.5, k2=1.0, num_values=20,
                                                 kbinningCase=ps.PS_BIN_GIVEN, dcosTheta=0.1)
        B64, N64, _, _ = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
        B32, N32, kap, _ = ctx.batch(cfgs, ps.PS_FP32_BATCHED, kappa=True)
    assert len(B32) == 20
    p = ora.RunParams(grid_size=n, box_size=box, which_field=1, use_only_phase=0, n=3, equilateral=0, k1=0.5,
                      k2=1.0, num_values=20, kbinwidth=1.0, kbinning=2, dcos_theta=0.1)
    ref = ora.ora_run(p, None, xhii)
    assert len(ref.B) == 20
    np.testing.assert_array_equal(k, ref.k)
    np.testing.assert_array_equal(N32, np.rint(ref.npoly))
    assert np.all(np.rint(ref.npoly) > 0)
    rel64 = np.abs(B64 - ref.B) / np.abs(ref.B)
    rel32 = np.abs(B32 - ref.B) / np.abs(ref.B)
    assert rel64.max() <= 1e-9, rel64
    assert rel32.max() <= 1e-5, (rel32, kap)


def _torch_lognormal(n, alpha, seed):
    """synth.lognormal_density's recipe, drawn on the GPU: white noise,
    amplitude sqrt(k^-alpha) up to Nyquist, unit variance, exp(g - 1/2) - 1."""
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    w = torch.randn((n, n, n), generator=gen, device="cuda", dtype=torch.float32)
    wk = torch.fft.rfftn(w)
    del w
    f = torch.fft.fftfreq(n, device="cuda") * n
    fz = torch.fft.rfftfreq(n, device="cuda") * n
    k2 = f[:, None, None] ** 2 + f[None, :, None] ** 2 + fz[None, None, :] ** 2
    amp = torch.where((k2 > 0) & (k2 <= (n / 2) ** 2), k2.clamp(min=1.0) ** (-alpha / 4.0), torch.zeros_like(k2))
    wk *= amp
    del amp, k2
    g = torch.fft.irfftn(wk, s=(n, n, n))
    del wk
    g = (g - g.mean()) / g.std()
    return (torch.exp(g.double() - 0.5) - 1.0).float()


def test_config_1024_power_and_triangles(gpu_lib):
    import torch
    ps = gpu_lib
    n, box = 1024, 1000.0
    field = _torch_lognormal(n, 1.5, 8)
    assert torch.isfinite(field).all()
    pk, _, _ = ps.read_params_to_kvectors(n, box, 2, num_values=2)
    eq, _, _ = ps.read_params_to_kvectors(n, box, 3, equilateral=1, num_values=64)
    iso, _, _ = ps.read_params_to_kvectors(n, box, 3, k1=0.3, k2=0.3, num_values=64)
    assert len(pk) == n // 2
    tri = [eq[i] for i in range(len(eq))] + [iso[i] for i in range(len(iso))]
    with ps.Context(n, box, methods=ps.PS_FP32_BATCHED) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_DENS, field)
        plan = ctx.plan([pk[i] for i in range(len(pk))] + tri)
        B32, N32, _, _ = plan.execute()
        plan.close()
    sample = list(range(0, 64, 9)) + list(range(64, 128, 9))
    sub = [pk[i] for i in range(len(pk))] + [tri[i] for i in sample]
    with ps.Context(n, box, methods=ps.PS_FP64_PLAIN) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_DENS, field.double())
        B64, N64, _, _ = ctx.batch(sub, ps.PS_FP64_PLAIN)
    got_B = np.concatenate([B32[: n // 2], B32[n // 2:][sample]])
    got_N = np.concatenate([N32[: n // 2], N32[n // 2:][sample]])
    has = np.rint(N64) != 0
    ok, rel = _close(got_B[has], B64[has], 1e-5, 1e-6)
    assert ok, rel.max()
    np.testing.assert_array_equal(got_N, np.rint(N64))
    assert np.all(N32[: n // 2] > 0)  # every shell below Nyquist holds modes


@pytest.mark.parametrize("n", [300, 600])
def test_config_mixed_radix_grid(gpu_lib, ora, n):
    """300^3 and 600^3 grids (2^a 3 5^2 cells, the sizes of the reference's
    accuracy study linked from its README): an XHI_DENS field in a box of
    n Mpc/h (ionised spheres at the benchmark's number density, lognormal
    density), phase-only, DERIVED binning, a 16-bin theta sweep with
    k1 = 0.3, k2 = 0.6 h/Mpc.  Batched FP32 against plain FP64 on every bin
    (1e-5 relative, no absolute floor; counts exact; DERIVED ranges
    identical); at 300^3 two bins also against the oracle."""
    ps = gpu_lib
    box = float(n)
    dens, xhii = synth.xhi_dens_inputs(n, box, int(round(32000 * (box / 400.0) ** 3)), 3, 2.0, 4)
    cfgs, k, th = ps.read_params_to_kvectors(n, box, 3, k1=0.3, k2=0.6, num_values=16,
                                             kbinningCase=ps.PS_BIN_DERIVED)
    with ps.Context(n, box) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        B64, N64, _, o64 = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
        B32, N32, kap, o32 = ctx.batch(cfgs, ps.PS_FP32_BATCHED, kappa=True)
    np.testing.assert_array_equal(N32, np.rint(N64))
    assert np.all(N32 > 0)
    rel = np.abs(B32 - B64) / np.abs(B64)
    assert rel.max() <= 1e-5, (rel, kap)
    for q in range(16):
        for l in range(3):
            assert o32[q].kmin[l] == o64[q].kmin[l] and o32[q].kmax[l] == o64[q].kmax[l]
    if n == 300:
        p = ora.RunParams(grid_size=n, box_size=box, which_field=2, use_only_phase=1, n=3, equilateral=0,
                          k1=0.3, k2=0.6, num_values=16, kbinwidth=1.0, kbinning=1)
        for t in (3, 11):
            ref = ora.ora_run(p, dens, xhii, max_cfg=1, first=t)
            assert abs(B64[t] - ref.B[0]) <= 1e-9 * abs(ref.B[0]), (t, B64[t], ref.B[0])
            assert abs(B32[t] - ref.B[0]) <= 1e-5 * abs(ref.B[0]), (t, B32[t], ref.B[0])
            assert N32[t] == np.rint(ref.npoly[0])
            np.testing.assert_array_equal([o32[t].kmin[l] for l in range(3)], ref.kmin[0])
            np.testing.assert_array_equal([o32[t].kmax[l] for l in range(3)], ref.kmax[0])
