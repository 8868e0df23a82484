"""Adjoint dB/d(delta) (ps_gpu_grad, no reference counterpart) against central
finite differences of the estimator itself, in FP64 (PS_FP64_PLAIN), and the
FP32 gradient against the FP64 one.

Tolerances: finite differences (eps = 1e-3) agree with the FP64 gradient to
1e-4 of max|grad| per voxel and 1e-4 relative per directional derivative; the
FP32 gradient agrees with the FP64 one to 1e-4 of max|grad|."""
import numpy as np
import pytest

from polyspectrum_b200 import synth

pytestmark = pytest.mark.gpu

EPS = 1e-3


def _B(ps, ctx, field, cfg, method):
    ctx.get_FT_field(ps.PS_FIELD_DENS, field, use_only_phase=0)
    return ctx.batch([cfg], method)[0][0]


def _grad(ps, ctx, field, cfg, method, double=True):
    ctx.get_FT_field(ps.PS_FIELD_DENS, field, use_only_phase=0)
    n = cfg.n
    return ctx.grad(n, [cfg.k[i] for i in range(n)], [cfg.kmin[i] for i in range(n)],
                    [cfg.kmax[i] for i in range(n)], cfg.kbinwidth, cfg.kbinningCase,
                    method=method, double=double)


def _fd_check(ps, n_grid, box, cfg, nvox=16, ndir=4, seed_vox=6, seed_dir=7, field_seed=5):
    field = synth.lognormal_density(n_grid, 2.0, field_seed).astype(np.float64)
    with ps.Context(n_grid, box, methods=ps.PS_FP64_PLAIN) as ctx:
        g = _grad(ps, ctx, field, cfg, ps.PS_FP64_PLAIN)
        gmax = np.abs(g).max()
        assert gmax > 0
        rng = np.random.default_rng(seed_vox)
        vox = rng.integers(0, n_grid, size=(nvox, 3))
        for v in vox:
            fp = field.copy()
            fm = field.copy()
            fp[tuple(v)] += EPS
            fm[tuple(v)] -= EPS
            fd = (_B(ps, ctx, fp, cfg, 1) - _B(ps, ctx, fm, cfg, 1)) / (2 * EPS)
            assert abs(fd - g[tuple(v)]) <= 1e-4 * gmax, (v, fd, g[tuple(v)], gmax)
        rng = np.random.default_rng(seed_dir)
        for _ in range(ndir):
            d = rng.standard_normal(field.shape)
            d /= np.linalg.norm(d)
            fd = (_B(ps, ctx, field + EPS * d, cfg, 1) - _B(ps, ctx, field - EPS * d, cfg, 1)) / (2 * EPS)
            an = float((g * d).sum())
            assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-300) + 1e-6 * gmax, (fd, an)
    return g


@pytest.mark.parametrize("kb", [0, 1, 2, 3])
def test_grad_theta_config_fd(gpu_lib, kb):
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=3.2 * kf, k2=4.1 * kf, num_values=5,
                                            kbinningCase=kb, dcosTheta=0.2)
    _fd_check(ps, n_grid, box, cfgs[2])


def test_grad_equilateral_fd(gpu_lib):
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    cfg = ps.make_cfg(3, [4.2 * kf] * 3, kbinwidth=1.0)
    _fd_check(ps, n_grid, box, cfg)


def test_grad_power_spectrum_fd(gpu_lib):
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    cfg = ps.make_cfg(2, [5.0 * kf] * 2, kbinwidth=1.0)
    _fd_check(ps, n_grid, box, cfg)


def test_grad_fp32_matches_fp64(gpu_lib):
    ps = gpu_lib
    n_grid, box = 64, 150.0
    kf = 2 * np.pi / box
    field = synth.lognormal_density(n_grid, 2.0, 9).astype(np.float32)
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=4.5 * kf, k2=6.1 * kf, num_values=4,
                                            kbinningCase=1)
    with ps.Context(n_grid, box) as ctx:
        for q in range(len(cfgs)):
            g64 = _grad(ps, ctx, field, cfgs[q], ps.PS_FP64_PLAIN)
            g32 = _grad(ps, ctx, field, cfgs[q], ps.PS_FP32_BATCHED, double=False)
            assert np.abs(g32 - g64).max() <= 1e-4 * np.abs(g64).max()


def test_grad_refuses_phase_only(gpu_lib):
    ps = gpu_lib
    field = synth.lognormal_density(16, 2.0, 1)
    with ps.Context(16, 100.0) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_DENS, field, use_only_phase=1)
        with pytest.raises(ps.PsError) as e:
            ctx.grad(2, [0.2, 0.2], [0, 0], [0, 0], 1.0, 0)
        assert e.value.status == -7


def test_torch_autograd_binding(gpu_lib):
    import torch

    from polyspectrum_b200.autograd import polyspectrum
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    f = torch.from_numpy(synth.lognormal_density(n_grid, 2.0, 3).astype(np.float64)).cuda()
    f.requires_grad_(True)
    cfg = ps.make_cfg(3, [3.3 * kf, 4.0 * kf, 5.1 * kf], kbinwidth=1.0)
    with ps.Context(n_grid, box, methods=ps.PS_FP64_PLAIN) as ctx:
        B = polyspectrum(f, ctx, cfg)
        (2.0 * B).backward()
        g = _grad(ps, ctx, f.detach().cpu().numpy(), cfg, ps.PS_FP64_PLAIN)
    np.testing.assert_allclose(f.grad.cpu().numpy(), 2.0 * g, rtol=0, atol=1e-12 * np.abs(g).max())


def test_grad_equilateral_256(gpu_lib):
    """The 256^3 gradient configuration: DENS (P ~ k^-2), equilateral k = 0.8 h/Mpc, kbinwidth 1,
    DEFAULT binning; central differences (eps 1e-3, FP64) on 64 seeded voxels and 8 random
    directions; FP32 gradient against FP64."""
    ps = gpu_lib
    n_grid, box = 256, 200.0
    cfg = ps.make_cfg(3, [0.8] * 3, kbinwidth=1.0)
    g64 = _fd_check(ps, n_grid, box, cfg, nvox=64, ndir=8, seed_vox=6, seed_dir=7, field_seed=5)
    field = synth.lognormal_density(n_grid, 2.0, 5).astype(np.float32)
    with ps.Context(n_grid, box, methods=ps.PS_FP32_BATCHED) as ctx:
        g32 = _grad(ps, ctx, field, cfg, ps.PS_FP32_BATCHED, double=False)
    assert np.abs(g32 - g64).max() <= 1e-4 * np.abs(g64).max()


def _fd_check_phase(ps, n_grid, box, cfg, nvox=12, ndir=4, field_seed=5):
    """Phase-only field: the gradient through z/|z| against central differences."""
    field = synth.lognormal_density(n_grid, 2.0, field_seed).astype(np.float64)
    with ps.Context(n_grid, box, methods=ps.PS_FP64_PLAIN) as ctx:
        ctx.keep_modulus(True)

        def B(f):
            ctx.get_FT_field(ps.PS_FIELD_DENS, f, use_only_phase=1)
            return ctx.batch([cfg], 1)[0][0]
        ctx.get_FT_field(ps.PS_FIELD_DENS, field, use_only_phase=1)
        n = cfg.n
        g = ctx.grad(n, [cfg.k[i] for i in range(n)], [cfg.kmin[i] for i in range(n)],
                     [cfg.kmax[i] for i in range(n)], cfg.kbinwidth, cfg.kbinningCase, method=1)
        gmax = np.abs(g).max()
        assert gmax > 0
        rng = np.random.default_rng(6)
        for v in rng.integers(0, n_grid, size=(nvox, 3)):
            fp, fm = field.copy(), field.copy()
            fp[tuple(v)] += EPS
            fm[tuple(v)] -= EPS
            fd = (B(fp) - B(fm)) / (2 * EPS)
            assert abs(fd - g[tuple(v)]) <= 1e-4 * gmax, (v, fd, g[tuple(v)], gmax)
        rng = np.random.default_rng(7)
        for _ in range(ndir):
            d = rng.standard_normal(field.shape)
            d /= np.linalg.norm(d)
            fd = (B(field + EPS * d) - B(field - EPS * d)) / (2 * EPS)
            an = float((g * d).sum())
            assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-300) + 1e-6 * gmax, (fd, an)
    return g


@pytest.mark.parametrize("kb", [0, 1])
def test_grad_phase_only_fd(gpu_lib, kb):
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=3.2 * kf, k2=4.1 * kf, num_values=5,
                                            kbinningCase=kb)
    _fd_check_phase(ps, n_grid, box, cfgs[2])


def test_grad_phase_only_power_is_zero(gpu_lib):
    """Phase-only, n = 2: every mode has |phi|^2 = 1, so P(k) does not depend on
    the field and its gradient vanishes (rounding residue only)."""
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    field = synth.lognormal_density(n_grid, 2.0, 5).astype(np.float64)
    cfg = ps.make_cfg(2, [5.0 * kf] * 2, kbinwidth=1.0)
    with ps.Context(n_grid, box, methods=ps.PS_FP64_PLAIN) as ctx:
        ctx.keep_modulus(True)
        ctx.get_FT_field(ps.PS_FIELD_DENS, field, use_only_phase=1)
        B = ctx.batch([cfg], 1)[0][0]
        g = ctx.grad(2, [5.0 * kf] * 2, [0, 0], [0, 0], 1.0, 0, method=1)
    d = np.random.default_rng(3).standard_normal(field.shape)
    d *= np.linalg.norm(field) / np.linalg.norm(d)
    # a change of the field as large as the field itself moves B by ~0
    assert abs(float((g * d).sum())) <= 1e-9 * abs(B), (float((g * d).sum()), B)


def test_grad_phase_only_fp32_and_torch(gpu_lib):
    """FP32 phase-only gradient against FP64, and the torch binding with
    use_only_phase = 1 against the C-ABI gradient."""
    import torch

    from polyspectrum_b200.autograd import polyspectrum
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    cfg = ps.make_cfg(3, [3.3 * kf, 4.0 * kf, 5.1 * kf], kbinwidth=1.0)
    field = synth.lognormal_density(n_grid, 2.0, 3).astype(np.float64)
    grads = []
    for method, dbl in ((ps.PS_FP64_PLAIN, True), (ps.PS_FP32_BATCHED, False)):
        with ps.Context(n_grid, box, methods=method) as ctx:
            ctx.keep_modulus(True)
            ctx.get_FT_field(ps.PS_FIELD_DENS, field.astype(np.float64 if dbl else np.float32), use_only_phase=1)
            grads.append(ctx.grad(3, list(cfg.k)[:3], list(cfg.kmin)[:3], list(cfg.kmax)[:3], 1.0, 0,
                                  method=method, double=dbl))
    assert np.abs(grads[1] - grads[0]).max() <= 1e-4 * np.abs(grads[0]).max()
    f = torch.from_numpy(field).cuda().requires_grad_(True)
    with ps.Context(n_grid, box, methods=ps.PS_FP64_PLAIN) as ctx:
        B = polyspectrum(f, ctx, cfg, use_only_phase=1)
        B.backward()
    np.testing.assert_allclose(f.grad.cpu().numpy(), grads[0], rtol=0, atol=1e-12 * np.abs(grads[0]).max())
