"""GPU parity: the CUDA library through its C-ABI against the CPU oracle on
the same seeded inputs, for every binning case, n = 2 and 3, equilateral and
theta sweeps, phase-only on and off, and the three field kinds.

Tolerances (written here, checked per configuration):
  * PS_FP64_PLAIN  : |dB| <= 1e-9 |B| + 1e-11 max|B| of the sweep;
                     |dNpoly| <= 1e-7 max(1, Npoly)
  * PS_FP32_BATCHED: |dB| <= 1e-5 |B| + 1e-6 max|B| of the sweep
                     (the second term covers configurations whose sum cancels
                     to near zero, where a relative error has no meaning);
                     Npoly == round(Npoly_reference) exactly
  * DERIVED k ranges written back: bit-identical for both methods.
Configurations without any polygon (Npoly rounds to 0) have B = 0/0 in exact
arithmetic; the reference returns a ratio of rounding residues there, the
batched method NaN, so B is not compared for them.
"""
import numpy as np
import pytest

from _cases import field_args, fields, sweep_params

pytestmark = pytest.mark.gpu

TOL = {1: (1e-9, 1e-11), 2: (1e-5, 1e-6)}


def run_both(ps, ora, n_grid, box, case, method):
    dens, xhii = fields(n_grid, box)
    dd, xx = field_args(case["which_field"], dens, xhii)
    p = ora.RunParams(grid_size=n_grid, box_size=box, **case)
    ref = ora.ora_run(p, dd, xx)
    with ps.Context(n_grid, box, methods=method) as ctx:
        ctx.get_FT_field(case["which_field"], dd, xx, use_only_phase=case["use_only_phase"])
        got = ps.run_sweep(ctx, n_grid, box, case["n"], method=method,
                           equilateral=case["equilateral"], k1=case["k1"], k2=case["k2"],
                           num_values=case["num_values"], theta=case["theta"],
                           kbinwidth=case["kbinwidth"], kbinningCase=case["kbinning"],
                           dcosTheta=case["dcos_theta"])
    return ref, got


def check(ref, got, method, label=""):
    rt, at = TOL[method]
    np.testing.assert_array_equal(got.k, ref.k)
    scale = np.nanmax(np.abs(ref.B)) if np.isfinite(ref.B).any() else 0.0
    has = np.rint(ref.npoly) != 0
    err = np.abs(got.B - ref.B)
    bound = rt * np.abs(ref.B) + at * scale
    bad = has & ~(err <= bound)
    assert not bad.any(), f"{label} B mismatch: got {got.B[bad]} ref {ref.B[bad]}"
    if method == 2:
        np.testing.assert_array_equal(got.npoly, np.rint(ref.npoly), err_msg=label)
    else:
        assert np.all(np.abs(got.npoly - ref.npoly) <= 1e-7 * np.maximum(1, np.abs(ref.npoly))), label
        np.testing.assert_array_equal(np.rint(got.npoly), np.rint(ref.npoly), err_msg=label)


CASES = sweep_params(32, 200.0)


@pytest.mark.parametrize("method", [1, 2], ids=["plain64", "batched32"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "n{n}_eq{equilateral}_kb{kbinning}_ph{use_only_phase}_f{which_field}".format(**c))
def test_sweep_matches_oracle(gpu_lib, ora, case, method):
    ref, got = run_both(gpu_lib, ora, 32, 200.0, case, method)
    check(ref, got, method, str(case))
    if case["kbinning"] == 1:
        np.testing.assert_array_equal(got.kmin, ref.kmin)
        np.testing.assert_array_equal(got.kmax, ref.kmax)


@pytest.mark.parametrize("n_grid", [16, 64])
@pytest.mark.parametrize("method", [1, 2], ids=["plain64", "batched32"])
def test_other_grid_sizes(gpu_lib, ora, n_grid, method):
    box = 150.0
    kf = 2 * np.pi / box
    case = dict(n=3, equilateral=0, k1=2.7 * kf, k2=4.1 * kf, num_values=5, theta=0.0,
                kbinwidth=1.0, kbinning=1, dcos_theta=0.2, use_only_phase=0, which_field=2)
    ref, got = run_both(gpu_lib, ora, n_grid, box, case, method)
    check(ref, got, method)
    np.testing.assert_array_equal(got.kmin, ref.kmin)


@pytest.mark.parametrize("bw", [0.5, 2.0, 3.0])
@pytest.mark.parametrize("kb", [0, 1, 2, 3])
def test_binwidths(gpu_lib, ora, bw, kb):
    box = 100.0
    kf = 2 * np.pi / box
    case = dict(n=3, equilateral=0, k1=3.0 * kf, k2=5.0 * kf, num_values=4, theta=0.0,
                kbinwidth=bw, kbinning=kb, dcos_theta=0.15, use_only_phase=0, which_field=0)
    for method in (1, 2):
        ref, got = run_both(gpu_lib, ora, 32, box, case, method)
        check(ref, got, method, f"bw={bw} kb={kb} m={method}")


def test_single_config_api(gpu_lib, ora):
    """ps_gpu_polyspectrum (one configuration, reference argument order)."""
    ps = gpu_lib
    n_grid, box = 32, 200.0
    dens, _ = fields(n_grid, box)
    L = float(np.float32(box))
    dk = ora.ora_forward(n_grid, 0, dens)
    kf = 2 * np.pi / box
    k = np.array([3.3 * kf, 4.2 * kf, 5.9 * kf])
    for kb in (0, 1, 2, 3):
        lo = np.array([0.0, 0.0, 5.0 * kf])
        hi = np.array([0.0, 0.0, 6.5 * kf])
        b_ref, _, _, lo_ref, hi_ref = ora.ora_polyspectrum(n_grid, dk, k, lo, hi, 1.0, kb, L)
        n_ref = ora.ora_num_polygons(n_grid, k, lo_ref, hi_ref, 1.0, kb, L)
        with ps.Context(n_grid, box, methods=ps.PS_FP64_PLAIN) as ctx:
            ctx.get_FT_field(0, dens)
            b, npol, lo2, hi2 = ctx.polyspectrum(3, k, lo, hi, 1.0, kb)
        assert abs(b - b_ref) <= 1e-9 * abs(b_ref)
        assert abs(npol - n_ref) <= 1e-7 * max(1.0, n_ref)
        np.testing.assert_array_equal(lo2, lo_ref)
        np.testing.assert_array_equal(hi2, hi_ref)


def test_derived_n2_is_refused(gpu_lib):
    ps = gpu_lib
    with ps.Context(16, 100.0) as ctx:
        ctx.get_FT_field(0, fields(16, 100.0)[0])
        cfg = ps.make_cfg(2, [0.2, 0.2], [0.2, 0.2], [0.2, 0.2], 1.0, ps.PS_BIN_DERIVED)
        for method in (1, 2):
            with pytest.raises(ps.PsError) as e:
                ctx.batch([cfg], method)
            assert e.value.status == -8


def test_device_resident_field(gpu_lib, ora):
    """Field pointers in device memory (torch tensors) give the same result."""
    import torch
    ps = gpu_lib
    n_grid, box = 32, 200.0
    dens, xhii = fields(n_grid, box)
    dd, xx = field_args(2, dens, xhii)
    cfgs, k, th = ps.read_params_to_kvectors(n_grid, box, 3, k1=0.1, k2=0.13, num_values=4,
                                             kbinningCase=1)
    outs = []
    for mem in ("host", "device"):
        with ps.Context(n_grid, box) as ctx:
            if mem == "host":
                ctx.get_FT_field(2, dd, xx)
            else:
                ctx.get_FT_field(2, torch.from_numpy(dd).cuda(), torch.from_numpy(xx).cuda())
            outs.append(ctx.batch(cfgs, ps.PS_FP32_BATCHED)[:2])
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("method", [1, 2], ids=["plain64", "batched32"])
def test_condition_numbers(gpu_lib, method):
    """kappa = sum|terms| / |sum terms| of the final sum: >= 1, finite, and 1 for
    power spectra (all terms |dk|^2) in the batched method."""
    ps = gpu_lib
    n_grid, box = 32, 200.0
    dens, xhii = fields(n_grid, box)
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=0.1, k2=0.14, num_values=5, kbinningCase=1)
    with ps.Context(n_grid, box) as ctx:
        ctx.get_FT_field(0, dens)
        B, Np, kap, _ = ctx.batch(cfgs, method, kappa=True)
        assert np.all(np.isfinite(kap)) and np.all(kap >= 1.0 - 1e-12), kap
        p2, _, _ = ps.read_params_to_kvectors(n_grid, box, 2, num_values=2)
        _, _, kap2, _ = ctx.batch(p2, method, kappa=True)
        if method == 2:
            assert np.all(kap2 == 1.0)
        else:
            assert np.all(kap2 >= 1.0 - 1e-12)


def test_power_spectrum_sweep_many_shells(gpu_lib, ora):
    """n = 2 over all N/2 shells (several Parseval passes of 16) at 64^3."""
    ps = gpu_lib
    n_grid, box = 64, 300.0
    dens, _ = fields(n_grid, box)
    case = dict(n=2, equilateral=0, k1=0.0, k2=0.0, num_values=2, theta=0.0, kbinwidth=1.0,
                kbinning=0, dcos_theta=0.2, use_only_phase=0, which_field=0)
    for method in (1, 2):
        ref, got = run_both(ps, ora, n_grid, box, case, method)
        assert len(got.k) == n_grid // 2
        check(ref, got, method, f"pk m={method}")


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_plan_replay_matches_batch(gpu_lib, graph):
    """A plan (optionally captured into a CUDA graph on first execution)
    executed on two different fields gives, on each, exactly what an eager
    batch gives, including the DERIVED write-back."""
    ps = gpu_lib
    n_grid, box = 32, 200.0
    d1, x1 = fields(n_grid, box)
    d2, x2 = fields(n_grid, box, seed=7)
    cfgs = []
    for k1, k2 in ((0.1, 0.14), (0.12, 0.2)):
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=5, kbinningCase=1)
        cfgs += [c[i] for i in range(len(c))]
    eq, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, equilateral=1, num_values=3)
    p2, _, _ = ps.read_params_to_kvectors(n_grid, box, 2, num_values=2)
    cfgs += [eq[i] for i in range(len(eq))] + [p2[i] for i in range(len(p2))]
    with ps.Context(n_grid, box) as ctx:
        plan = ctx.plan(cfgs, graph=graph, kappa=True)
        for dens, xhii in ((d1, x1), (d2, x2), (d1, x1)):
            dd, xx = field_args(2, dens, xhii)
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            Bp, Np, kp, out = plan.execute()
            Be, Ne, ke, arr = ctx.batch(cfgs, ps.PS_FP32_BATCHED, kappa=True)
            np.testing.assert_array_equal(Bp, Be)
            np.testing.assert_array_equal(Np, Ne)
            np.testing.assert_array_equal(kp, ke)
            for i in range(len(cfgs)):
                assert list(out[i].kmin)[:3] == list(arr[i].kmin)[:3]
                assert list(out[i].kmax)[:3] == list(arr[i].kmax)[:3]
        plan.close()


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_prepared_plan_matches_batch(gpu_lib, graph):
    """ps_gpu_plan_prepare queued before the field load (the DERIVED chain and
    the exact counts on the side stream, overlapping the load) gives exactly
    the eager batch's results on every field, through execute, submit and
    launch; so do two plans prepared and executed in the opposite order, a
    prepare repeated, a prepared plan executed with per-kernel profiling on
    (eager on one lane) and a prepared plan counting with FP64 transforms."""
    import torch
    ps = gpu_lib
    n_grid, box = 32, 200.0
    d1, x1 = fields(n_grid, box)
    d2, x2 = fields(n_grid, box, seed=7)
    cfgs = []
    for k1, k2 in ((0.1, 0.14), (0.12, 0.2)):
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=5, kbinningCase=1)
        cfgs += [c[i] for i in range(len(c))]
    eq, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, equilateral=1, num_values=3)
    p2, _, _ = ps.read_params_to_kvectors(n_grid, box, 2, num_values=2)
    cfgs += [eq[i] for i in range(len(eq))] + [p2[i] for i in range(len(p2))]
    other = cfgs[:5]
    with ps.Context(n_grid, box) as ctx:
        plan = ctx.plan(cfgs, graph=graph, kappa=True)
        plan_b = ctx.plan(other, graph=graph)
        plan_f = ctx.plan(cfgs, graph=graph, fft_counts=True)

        def expect(dens, xhii, cf, kap=True):
            dd, xx = field_args(2, dens, xhii)
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            return ctx.batch(cf, ps.PS_FP32_BATCHED, kappa=kap)

        def same(got, ref, n):
            np.testing.assert_array_equal(got[0], ref[0])
            np.testing.assert_array_equal(got[1], ref[1])
            if got[2] is not None and ref[2] is not None:
                np.testing.assert_array_equal(got[2], ref[2])
            for i in range(n):
                assert list(got[3][i].kmin)[:3] == list(ref[3][i].kmin)[:3]
                assert list(got[3][i].kmax)[:3] == list(ref[3][i].kmax)[:3]

        for dens, xhii in ((d1, x1), (d2, x2), (d1, x1)):
            ref = expect(dens, xhii, cfgs)
            dd, xx = field_args(2, dens, xhii)
            # execute
            plan.prepare()
            plan.prepare()  # already prepared: no-op
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            same(plan.execute(), ref, len(cfgs))
            # launch, results read later
            plan.prepare()
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            plan.launch()
            same(plan.results(), ref, len(cfgs))
            # two plans prepared, executed in the opposite order
            ref_b = expect(dens, xhii, other, kap=False)
            plan.prepare()
            plan_b.prepare()
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            same(plan_b.execute(), ref_b, len(other))
            same(plan.execute(), ref, len(cfgs))
            # prepared, then executed with per-kernel profiling on
            plan.prepare()
            ctx.set_profiling(True)
            try:
                same(plan.execute(), ref, len(cfgs))
            finally:
                ctx.set_profiling(False)
            # FP64 transform counts, prepared
            plan_f.prepare()
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            got = plan_f.execute()
            same((got[0], got[1], None, got[3]), (ref[0], ref[1], None, ref[3]), len(cfgs))
        torch.cuda.synchronize()
        plan.close()
        plan_b.close()
        plan_f.close()


@pytest.mark.parametrize("pinned", [False, True], ids=["pageable", "pinned"])
def test_async_pipeline_matches_sync(gpu_lib, pinned):
    """Fields uploaded with set_field_async and plans submitted without waiting
    (uploads of the next field overlapping the current configurations) give,
    per field, exactly the synchronous results, DERIVED write-back and
    condition numbers included."""
    import torch
    ps = gpu_lib
    n_grid, box = 32, 200.0
    flds = [fields(n_grid, box), fields(n_grid, box, seed=7), fields(n_grid, box, seed=11)]
    cfgs = []
    for k1, k2 in ((0.1, 0.14), (0.12, 0.2)):
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=5, kbinningCase=1)
        cfgs += [c[i] for i in range(len(c))]
    p2, _, _ = ps.read_params_to_kvectors(n_grid, box, 2, num_values=2)
    cfgs += [p2[i] for i in range(len(p2))]
    args = []
    for dens, xhii in flds:
        dd, xx = field_args(2, dens, xhii)
        if pinned:
            dd, xx = torch.from_numpy(dd).pin_memory(), torch.from_numpy(xx).pin_memory()
        args.append((dd, xx))
    with ps.Context(n_grid, box, methods=ps.PS_FP32_BATCHED) as ctx:
        plan = ctx.plan(cfgs, graph=True, kappa=True)
        want = []
        for dd, xx in args:
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            want.append(plan.execute())
        subs = []
        order = [0, 1, 2, 1, 0, 2]
        for f in order:
            ctx.set_field_async(2, *args[f], use_only_phase=1)
            subs.append(plan.submit())
        ctx.synchronize()
        for f, sub in zip(order, subs):
            B, Np, kap, out = want[f]
            np.testing.assert_array_equal(sub.B, B)
            np.testing.assert_array_equal(sub.npoly, Np)
            np.testing.assert_array_equal(sub.kappa, kap)
            for i in range(len(cfgs)):
                assert list(sub.cfgs[i].kmin)[:3] == list(out[i].kmin)[:3]
                assert list(sub.cfgs[i].kmax)[:3] == list(out[i].kmax)[:3]
        plan.close()


def test_plan_outliving_context(gpu_lib):
    """Closing the context first leaves the plan destroyable and unusable."""
    ps = gpu_lib
    ctx = ps.Context(16, 100.0)
    ctx.get_FT_field(0, fields(16, 100.0)[0])
    cfgs, _, _ = ps.read_params_to_kvectors(16, 100.0, 3, k1=0.2, k2=0.3, num_values=3)
    plan = ctx.plan(cfgs)
    plan.execute()
    n0 = ctx.launch_count()
    plan.execute()
    assert ctx.launch_count() > n0
    ctx.close()
    plan.close()


@pytest.mark.parametrize("kb", [0, 1, 2, 3])
@pytest.mark.parametrize("n_grid", [64, 128])
def test_subgrid_groups_match_oracle(gpu_lib, ora, n_grid, kb):
    """Theta sweeps whose legs and closing shells are small against the grid run
    their pair group on a smaller alias-free grid (16 or 32 points for these
    shells); results match the oracle's N-grid sums, counts exactly."""
    box = 200.0
    kf = 2 * np.pi / box
    case = dict(n=3, equilateral=0, k1=2.2 * kf, k2=3.6 * kf, num_values=7, theta=0.0, kbinwidth=1.0,
                kbinning=kb, dcos_theta=0.2, use_only_phase=1, which_field=2)
    ref, got = run_both(gpu_lib, ora, n_grid, box, case, 2)
    check(ref, got, 2, f"N={n_grid} kb={kb}")
    if kb == 1:
        np.testing.assert_array_equal(got.kmin, ref.kmin)
        np.testing.assert_array_equal(got.kmax, ref.kmax)


@pytest.mark.parametrize("n_grid,pairs", [(256, [(0.5, 0.8)]), (512, [(0.8, 1.2), (1.0, 1.5)])],
                         ids=["N256_subgrid192", "N512_subgrid320_384"])
def test_mixed_radix_subgrids_match_plain(gpu_lib, n_grid, pairs):
    """DERIVED theta sweeps of the bench workload whose pair groups run on
    192-, 320- and 384-point sub-grids (radix-3 and radix-5 transforms): the
    batched FP32 method against the plain FP64 method (the reference dataflow
    on the full grid) on the same XHI_DENS phase field, B within the batched
    tolerance, counts and derived ranges identical."""
    from polyspectrum_b200 import synth
    ps = gpu_lib
    box = 400.0
    dens, xhii = synth.xhi_dens_inputs(n_grid, box, int(round(32000 * (n_grid / 512) ** 3)), 3, 2.0, 4)
    cfgs = []
    for k1, k2 in pairs:
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=16,
                                             kbinningCase=ps.PS_BIN_DERIVED)
        cfgs += [c[i] for i in range(len(c))]
    with ps.Context(n_grid, box) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        B32, N32, _, out32 = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
        B64, N64, _, out64 = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
    scale = np.abs(B64).max()
    assert np.all(np.abs(B32 - B64) <= 1e-5 * np.abs(B64) + 1e-6 * scale), (B32, B64)
    np.testing.assert_array_equal(N32, np.rint(N64))
    for i in range(len(cfgs)):
        assert list(out32[i].kmin)[:3] == list(out64[i].kmin)[:3]
        assert list(out32[i].kmax)[:3] == list(out64[i].kmax)[:3]


def test_autotuned_plan_and_tune_table(gpu_lib):
    """An autotuned plan (transform size per pair group and Y pass geometry
    per transform size picked by timing) keeps
    counts and derived ranges identical and B within the batched tolerance of
    plain FP64; its choices exported from one context and imported into
    another reproduce its results bit for bit without timing."""
    from polyspectrum_b200 import synth
    ps = gpu_lib
    n_grid, box = 256, 400.0
    dens, xhii = synth.xhi_dens_inputs(n_grid, box, 4000, 3, 2.0, 4)
    cfgs = []
    for k1, k2 in ((0.2, 0.5), (0.5, 0.8), (0.8, 1.2)):
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=8, kbinningCase=1)
        cfgs += [c[i] for i in range(len(c))]
    with ps.Context(n_grid, box) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        plan = ctx.plan(cfgs, autotune=True)
        Bt, Nt, _, outt = plan.execute()
        plan.close()
        B64, N64, _, out64 = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
        table = ctx.tune_export()
    assert table.count("grid ") >= 2, table
    assert "pencil " in table, table  # the Y pass geometry per transform size
    assert "pair " in table, table  # the pair kernel variant per transform size
    assert "dot " in table, table  # the dot pass geometry per transform size
    scale = np.abs(B64).max()
    assert np.all(np.abs(Bt - B64) <= 1e-5 * np.abs(B64) + 1e-6 * scale)
    np.testing.assert_array_equal(Nt, np.rint(N64))
    for i in range(len(cfgs)):
        assert list(outt[i].kmin)[:3] == list(out64[i].kmin)[:3]
    with ps.Context(n_grid, box) as ctx2:
        ctx2.tune_import(table)
        assert ctx2.tune_export() == table
        ctx2.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        plan2 = ctx2.plan(cfgs)
        B2, N2, _, _ = plan2.execute()
        plan2.close()
        with pytest.raises(ps.PsError):
            ctx2.tune_import("grid 256 1 2 three 64\n")
    np.testing.assert_array_equal(B2, Bt)
    np.testing.assert_array_equal(N2, Nt)


def test_pair_kernel_variants_from_tune_table(gpu_lib):
    """Every pair kernel variant the autotuner chooses from (0 the default,
    1 one live row transform, 2 twice the elements per thread) and both dot
    pass geometries (1: twice the elements per thread, with pair variants 1
    and 2), forced through an imported tune table on 128-, 192- and 256-point
    sub-grids, keep counts and derived ranges identical and B within the
    batched tolerance of plain FP64; a table naming a variant outside its
    range is refused."""
    from polyspectrum_b200 import synth
    ps = gpu_lib
    n_grid, box = 256, 400.0
    dens, xhii = synth.xhi_dens_inputs(n_grid, box, 4000, 3, 2.0, 4)
    cfgs = []
    for k1, k2 in ((0.2, 0.5), (0.5, 0.8), (0.8, 1.2)):
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=6, kbinningCase=1)
        cfgs += [c[i] for i in range(len(c))]
    with ps.Context(n_grid, box) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        plan = ctx.plan(cfgs, autotune=True)
        plan.close()
        grids = [ln.split() for ln in ctx.tune_export().splitlines() if ln.startswith("grid ")]
        B64, N64, _, out64 = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
    assert grids
    scale = np.abs(B64).max()
    for M in (128, 192, 256):
        table = "".join(f"grid {g[1]} {g[2]} {g[3]} {g[4]} {max(M, int(g[5]))}\n" for g in grids)
        for v in (0, 1, 2):
            with ps.Context(n_grid, box) as ctx:
                ctx.tune_import(table + "".join(f"pair {m} {v}\ndot {m} {int(v > 0)}\n" for m in (128, 192, 256)))
                assert f"pair {M} {v}" in ctx.tune_export()
                assert f"dot {M} {int(v > 0)}" in ctx.tune_export()
                ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
                plan = ctx.plan(cfgs)
                Bv, Nv, _, outv = plan.execute()
                plan.close()
            err = np.abs(Bv - B64)
            assert np.all(err <= 1e-5 * np.abs(B64) + 1e-6 * scale), (M, v, err.max())
            np.testing.assert_array_equal(Nv, np.rint(N64))
            for i in range(len(cfgs)):
                assert list(outv[i].kmin)[:3] == list(out64[i].kmin)[:3]
                assert list(outv[i].kmax)[:3] == list(out64[i].kmax)[:3]
    with ps.Context(n_grid, box) as ctx:
        with pytest.raises(ps.PsError):
            ctx.tune_import("pair 256 3\n")
        with pytest.raises(ps.PsError):
            ctx.tune_import("dot 256 2\n")


@pytest.mark.parametrize("legs", [(3.1, 4.2, 3.7, 5.0), (4.0, 4.0, 4.0, 4.0), (2.9, 3.6, 4.4, 3.1, 5.2)],
                         ids=["n4", "n4_equal", "n5"])
def test_higher_polygons_match_oracle(gpu_lib, ora, legs):
    """n = 4 and 5 (the estimator takes any n, polyspectrum.c:72; only the
    reference's configuration generator stops at 3): both methods against the
    oracle's polyspectrum() / num_polygons() for DEFAULT binning, with a
    repeated shell folded into a power."""
    ps = gpu_lib
    n_grid, box = 32, 100.0
    kf = 2 * np.pi / box
    dens, _ = fields(n_grid, box)
    L = float(np.float32(box))
    k = np.array(legs) * kf
    n = len(k)
    dk = ora.ora_forward(n_grid, 0, dens)
    lo = np.zeros(n)
    hi = np.zeros(n)
    b_ref, _, _, _, _ = ora.ora_polyspectrum(n_grid, dk, k, lo, hi, 1.0, 0, L)
    n_ref = ora.ora_num_polygons(n_grid, k, lo, hi, 1.0, 0, L)
    assert n_ref > 0
    cfg = ps.make_cfg(n, list(k), kbinwidth=1.0)
    with ps.Context(n_grid, box) as ctx:
        ctx.get_FT_field(0, dens)
        B64, N64, _, _ = ctx.batch([cfg], ps.PS_FP64_PLAIN)
        B32, N32, _, _ = ctx.batch([cfg], ps.PS_FP32_BATCHED)
    assert abs(B64[0] - b_ref) <= 1e-9 * abs(b_ref)
    assert abs(N64[0] - n_ref) <= 1e-7 * max(1.0, n_ref)
    assert abs(B32[0] - b_ref) <= 1e-5 * abs(b_ref)
    assert N32[0] == np.rint(n_ref)


def test_band_limited_spectrum(gpu_lib):
    """A field loaded with a plan's spectrum band gives that plan bit-identical
    results; computations reaching modes beyond the band are refused; a full
    load afterwards serves them again."""
    ps = gpu_lib
    n_grid, box = 64, 300.0
    dens, xhii = fields(n_grid, box)
    dd, xx = field_args(2, dens, xhii)
    cfgs = []
    for k1, k2 in ((0.06, 0.09), (0.05, 0.12)):
        c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=6, kbinningCase=1)
        cfgs += [c[i] for i in range(len(c))]
    p2, _, _ = ps.read_params_to_kvectors(n_grid, box, 2, num_values=2)
    with ps.Context(n_grid, box) as ctx:
        plan = ctx.plan(cfgs)
        band = plan.band
        assert 0 < band < n_grid // 2
        ctx.get_FT_field(2, dd, xx, use_only_phase=1)
        full = plan.execute()
        ctx.set_spectrum_band(band)
        ctx.get_FT_field(2, dd, xx, use_only_phase=1)
        lim = plan.execute()
        np.testing.assert_array_equal(lim[0], full[0])
        np.testing.assert_array_equal(lim[1], full[1])
        with pytest.raises(ps.PsError):  # all n = 2 shells reach the Nyquist band
            ctx.batch(p2, ps.PS_FP32_BATCHED)
        with pytest.raises(ps.PsError):
            ctx.batch([p2[len(p2) - 1]], ps.PS_FP64_PLAIN)
        ctx.set_spectrum_band(-1)
        ctx.get_FT_field(2, dd, xx, use_only_phase=1)
        ctx.batch(p2, ps.PS_FP32_BATCHED)
        plan.close()


def test_plan_launch_and_results(gpu_lib):
    """Executions queued without read-back (ps_gpu_plan_launch) over several
    fields; ps_gpu_plan_results returns exactly the latest execution's
    results, DERIVED write-back included."""
    ps = gpu_lib
    n_grid, box = 32, 200.0
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=0.1, k2=0.14, num_values=5, kbinningCase=1)
    f1 = field_args(2, *fields(n_grid, box))
    f2 = field_args(2, *fields(n_grid, box, seed=7))
    with ps.Context(n_grid, box) as ctx:
        plan = ctx.plan(cfgs)
        ctx.get_FT_field(2, *f2, use_only_phase=1)
        want = plan.execute()
        for f in (f1, f2, f1, f2):
            ctx.set_field_async(2, *f, use_only_phase=1)
            plan.launch()
        B, Np, _, out = plan.results()
        ctx.synchronize()
        plan.close()
    np.testing.assert_array_equal(B, want[0])
    np.testing.assert_array_equal(Np, want[1])
    for i in range(len(cfgs)):
        assert list(out[i].kmin)[:3] == list(want[3][i].kmin)[:3]


@pytest.mark.parametrize("layout", ["xhidens_f32", "xhidens_mixed", "xhii_f64", "dens_f32"])
def test_field_files_match_set_field(gpu_lib, tmp_path, layout):
    """Grids streamed from raw files (ps_gpu_set_field_files: chunked through
    page-locked buffers, a float file beside a double one widened on the
    device) give exactly the results of the same grids passed as arrays; a
    short file is an I/O error."""
    ps = gpu_lib
    n_grid, box = 32, 200.0
    dens, xhii = fields(n_grid, box)
    dens = (1.0 + dens.astype(np.float64))
    which, d_dp, x_dp = {"xhidens_f32": (2, 0, 0), "xhidens_mixed": (2, 0, 1), "xhii_f64": (1, 0, 1),
                         "dens_f32": (0, 0, 0)}[layout]
    d_arr = dens if d_dp else dens.astype(np.float32)
    x_arr = xhii.astype(np.float64) if x_dp else xhii.astype(np.float32)
    d_arr.tofile(tmp_path / "dens.raw")
    x_arr.tofile(tmp_path / "xhii.raw")
    dp = (which != 1 and d_dp) or (which != 0 and x_dp)
    as_field = lambda a: a.astype(np.float64) if dp else a
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=0.1, k2=0.14, num_values=4, kbinningCase=1)
    with ps.Context(n_grid, box) as ctx:
        ctx.get_FT_field(which, as_field(d_arr) if which != 1 else None, as_field(x_arr) if which != 0 else None,
                         use_only_phase=1)
        want = [ctx.batch(cfgs, m)[:2] for m in (ps.PS_FP64_PLAIN, ps.PS_FP32_BATCHED)]
        ctx.set_field_files(which, str(tmp_path / "dens.raw") if which != 1 else None, d_dp,
                            str(tmp_path / "xhii.raw") if which != 0 else None, x_dp, use_only_phase=1)
        got = [ctx.batch(cfgs, m)[:2] for m in (ps.PS_FP64_PLAIN, ps.PS_FP32_BATCHED)]
        for (Bw, Nw), (Bg, Ng) in zip(want, got):
            np.testing.assert_array_equal(Bg, Bw)
            np.testing.assert_array_equal(Ng, Nw)
        short = tmp_path / "short.raw"
        d_arr.ravel()[:100].tofile(short)
        with pytest.raises(ps.PsError) as e:
            ctx.set_field_files(0, str(short), d_dp, None, 0, use_only_phase=1)
        assert e.value.status == -3


@pytest.mark.parametrize("methods", ["fp32_only", "both"])
def test_host_xhi_dens_composition(gpu_lib, methods):
    """Host float XHI_DENS inputs of an FP32-only context are composed on the
    host and uploaded as one float array (ps_gpu_upload_bytes = N^3 * 4);
    with both methods the two arrays go up (2 N^3 * 4).  Either way the
    results equal, bit for bit, those of the same arrays resident on the device
    (composed by the r2c loader), synchronous and asynchronous loads alike."""
    import torch
    ps = gpu_lib
    n_grid, box = 32, 200.0
    dens, xhii = field_args(2, *fields(n_grid, box))
    m = ps.PS_FP32_BATCHED if methods == "fp32_only" else ps.PS_FP32_BATCHED | ps.PS_FP64_PLAIN
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=0.1, k2=0.14, num_values=5, kbinningCase=1)
    with ps.Context(n_grid, box, methods=m) as ctx:
        ctx.get_FT_field(2, torch.from_numpy(dens).cuda(), torch.from_numpy(xhii).cuda(), use_only_phase=1)
        want = ctx.batch(cfgs, ps.PS_FP32_BATCHED)[:2]
        ctx.get_FT_field(2, dens, xhii, use_only_phase=1)
        assert ctx.upload_bytes() == n_grid ** 3 * 4 * (1 if methods == "fp32_only" else 2)
        got = ctx.batch(cfgs, ps.PS_FP32_BATCHED)[:2]
        ctx.set_field_async(2, dens, xhii, use_only_phase=1)
        ctx.synchronize()
        got_async = ctx.batch(cfgs, ps.PS_FP32_BATCHED)[:2]
        # page-locked inputs: part of the rows go up as they are, the rest composed
        dp, xp = torch.from_numpy(dens).pin_memory(), torch.from_numpy(xhii).pin_memory()
        got_pinned = []
        for _ in range(3):  # the split is re-balanced after every load
            ctx.set_field_async(2, dp, xp, use_only_phase=1)
            ctx.synchronize()
            up = ctx.upload_bytes()
            assert n_grid ** 3 * 4 <= up <= 2 * n_grid ** 3 * 4
            got_pinned.append(ctx.batch(cfgs, ps.PS_FP32_BATCHED)[:2])
    for g in [got, got_async] + got_pinned:
        np.testing.assert_array_equal(g[0], want[0])
        np.testing.assert_array_equal(g[1], want[1])


@pytest.mark.parametrize("n_grid", [48, 60, 96])
@pytest.mark.parametrize("method", [1, 2], ids=["plain64", "batched32"])
@pytest.mark.parametrize("kb", [0, 1, 2, 3])
def test_mixed_radix_grid_sizes(gpu_lib, ora, n_grid, method, kb):
    """Grids of 2^a 3^b 5^c cells other than powers of two (the reference's
    FFTW transforms any N, fft.c:30-36,50-56): 48 and 96 run the register
    passes with a radix-3 factor, 60 the shared-memory passes (odd part 15).
    A theta sweep of the XHI_DENS field in every binning case (phase-only with
    DERIVED binning), and the power spectrum over all shells."""
    box = 150.0
    kf = 2 * np.pi / box
    case = dict(n=3, equilateral=0, k1=3.3 * kf, k2=5.1 * kf, num_values=6, theta=0.0,
                kbinwidth=1.0, kbinning=kb, dcos_theta=0.2, use_only_phase=1 if kb == 1 else 0, which_field=2)
    ref, got = run_both(gpu_lib, ora, n_grid, box, case, method)
    check(ref, got, method, f"N={n_grid} kb={kb}")
    np.testing.assert_array_equal(got.kmin, ref.kmin)
    np.testing.assert_array_equal(got.kmax, ref.kmax)
    if kb == 0:
        p2 = dict(n=2, equilateral=0, k1=0.0, k2=0.0, num_values=2, theta=0.0, kbinwidth=1.0, kbinning=0,
                  dcos_theta=0.2, use_only_phase=0, which_field=0)
        ref, got = run_both(gpu_lib, ora, n_grid, box, p2, method)
        assert len(got.B) == n_grid // 2
        check(ref, got, method, f"N={n_grid} power spectrum")


def _plan_both_counts(ps, ctx, cfgs):
    """(B, Npoly) of a plan counting by enumeration and of one counting by
    FP64 unit-shell transforms."""
    out = []
    for fft in (False, True):
        plan = ctx.plan(cfgs, graph=False, fft_counts=fft)
        B, Np, _, _ = plan.execute()
        plan.close()
        out.append((B, Np))
    return out


@pytest.mark.parametrize("n_grid,k1,k2,kb", [(64, 4.3, 7.6, 1), (128, 9.1, 13.7, 1), (128, 6.2, 6.2, 2),
                                             (32, 9.2, 11.4, 1), (48, 8.7, 12.2, 0)])
def test_enumerated_counts_match_transforms(gpu_lib, ora, n_grid, k1, k2, kb):
    """Exact pair counts (integer enumeration over orbit representatives,
    the default for interval shells) equal the FP64 unit-shell transforms'
    rounded counts, and so do the B they normalise, bit for bit; the 32^3 case
    (k1 + k2 above N/2 fundamental modes) wraps sums around the grid as the
    reference's cyclic sums do, and is also checked against the oracle."""
    ps = gpu_lib
    box = 150.0
    kf = 2 * np.pi / box
    dens, xhii = fields(n_grid, box)
    dd, xx = field_args(2, dens, xhii)
    cfgs, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1 * kf, k2=k2 * kf, num_values=7,
                                            kbinningCase=kb, dcosTheta=0.2)
    with ps.Context(n_grid, box, methods=ps.PS_FP32_BATCHED) as ctx:
        ctx.get_FT_field(2, dd, xx, use_only_phase=0)
        (Be, Ne), (Bf, Nf) = _plan_both_counts(ps, ctx, cfgs)
    np.testing.assert_array_equal(Ne, Nf)
    np.testing.assert_array_equal(Be, Bf)
    if n_grid == 32:
        p = ora.RunParams(grid_size=n_grid, box_size=box, which_field=2, use_only_phase=0, n=3, equilateral=0,
                          k1=k1 * kf, k2=k2 * kf, num_values=7, kbinwidth=1.0, kbinning=kb, dcos_theta=0.2)
        ref = ora.ora_run(p, dd, xx)
        np.testing.assert_array_equal(Ne, np.rint(ref.npoly))
