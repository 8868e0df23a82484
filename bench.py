#!/usr/bin/env python
"""Benchmark of the polyspectrum estimator: bispectrum configurations per
second on a 64-configuration theta sweep at 512^3.

Workload (one "step"): an XHI_DENS field (dens*(1 - xHII)) of 512^3 float32
cells in a 400 Mpc/h box - xHII from 32000 seeded ionised spheres, dens =
1 + lognormal delta (P ~ k^-2) - phase-only, DERIVED binning, kbinwidth 1;
four (k1, k2) sweeps {(0.2,0.5), (0.5,0.8), (0.8,1.2), (1.0,1.5)} h/Mpc of 16
theta bins each = 64 bispectrum configurations with their polygon counts.
A step runs the forward transform of the field and all 64 configurations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--save-tune FILE | --tune-table FILE]

Prints one JSON line (rank 0).  `value` is device-timed with inputs resident
in HBM; `e2e` is the same step through the C-ABI from pinned host inputs with
the host->device copies and the result read-back inside the timed region;
`parity` checks the timed results against plain FP64 (all 64) and the
reference (configuration 0).  With --gpus N > 1 (one process per GPU under
torchrun) the step is the sharded path with weak scaling: 64 configurations
per rank (the four sweeps once per rank, shifted by -0.005 r h/Mpc for copy
r), each rank's share one plan, one NCCL all-gather of the results per step;
--replicas runs N independent copies of the 64-configuration step instead.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bispectrum configs/s @512^3 batched-FP32 vs plain FP64-GPU, rel err<=1e-5"
UNIT = "configs/s"
PAIRS = [(0.2, 0.5), (0.5, 0.8), (0.8, 1.2), (1.0, 1.5)]


def workload(grid: int):
    return dict(workload=f"xhi_dens_{grid}^3_phase_derived_theta_sweep_64cfg", grid=grid, box=400.0,
                spheres=int(round(32000 * (grid / 512) ** 3)), seed_ion=3, alpha=2.0, seed_dens=4,
                pairs=PAIRS, num_values=16, binning="DERIVED", kbinwidth=1.0, use_only_phase=1)


def make_inputs(w):
    from polyspectrum_b200 import synth
    dens, xhii = synth.xhi_dens_inputs(w["grid"], w["box"], w["spheres"], w["seed_ion"], w["alpha"],
                                       w["seed_dens"])
    return dens, xhii


def make_cfgs(ps, w, copies: int = 1):
    """The workload's configurations; with copies > 1 the four sweeps again
    per copy r, both legs shifted by -0.005 r h/Mpc (distinct shells of about
    the same cost: the multi-GPU workload of 64 configurations per rank)."""
    import ctypes as C
    allc = []
    pairs = [(k1 - 0.005 * r, k2 - 0.005 * r) for r in range(copies) for k1, k2 in w["pairs"]]
    for k1, k2 in pairs:
        cfgs, _, _ = ps.read_params_to_kvectors(w["grid"], w["box"], 3, k1=k1, k2=k2,
                                                num_values=w["num_values"],
                                                kbinningCase=ps.PS_BIN_DERIVED)
        allc += [cfgs[i] for i in range(len(cfgs))]
    arr = (ps.ps_cfg * len(allc))()
    for i, g in enumerate(allc):
        C.memmove(C.byref(arr[i]), C.byref(g), C.sizeof(ps.ps_cfg))
    return arr


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples (every 50 ms) read by a thread,
    each stamped with the host clock, so that a window of the run (the timed
    regions) can be summarised."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: str):
        import threading
        self.rows = []
        self.proc = None
        self.ready = threading.Event()
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", index], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                self.rows.append((time.time(), dict(sm=float(f[1]), smax=float(f[2]), power=float(f[3]),
                                                    hw=f[5], hwt=f[6], swt=f[7], swp=f[8])))
                self.ready.set()
            except ValueError:
                continue

    def wait_ready(self, timeout: float = 10.0):
        if self.proc:
            self.ready.wait(timeout)

    def close(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, windows):
        """Summary of the samples taken inside the [t0, t1] host-clock windows."""
        if not self.proc:
            return None
        rows = [r for t, r in list(self.rows) if any(t0 <= t <= t1 + 0.06 for t0, t1 in windows)]
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return dict(sm_mhz=float(np.median([r["sm"] for r in rows])), sm_max_mhz=rows[0]["smax"],
                    reasons=sorted(reasons), samples=len(rows),
                    power_w_max=max(r["power"] for r in rows))


def gpu_index(local_rank: int) -> str:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        parts = [p.strip() for p in vis.split(",") if p.strip()]
        if local_rank < len(parts):
            return parts[local_rank]
    return str(local_rank)


# --------------------------------------------------------------------------- CPU
def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference_sample(w, dens, xhii, first: int = 0, count: int = 1, threads: int | None = None):
    """Time the reference's CPU implementation on `count` configurations of the
    workload.  Uses oracle/_ref (the reference's own C, FFT shim) when built,
    else the oracle restatement.  `threads`: threads of the shim FFT (default:
    every CPU).  Returns (configs/s, kind, cores, sample, seconds, RunResult)."""
    import oracle
    k1, k2 = w["pairs"][0]
    p = oracle.RunParams(grid_size=w["grid"], box_size=w["box"], which_field=2,
                         use_only_phase=w["use_only_phase"], n=3, equilateral=0, k1=k1, k2=k2,
                         num_values=w["num_values"], kbinning=1, kbinwidth=w["kbinwidth"])
    cores = threads or os.cpu_count() or 1
    t0 = time.time()
    if oracle.ref_available():
        oracle.ref_set_threads(cores)
        r = oracle.ref_run(p, dens, xhii, first=first, count=count)
        kind = "reference"
        t_fwd, t_cfg = r.t_forward, r.t_configs
    else:
        oracle.ora_set_threads(cores)
        t_a = time.time()
        r = oracle.ora_run(p, dens, xhii, max_cfg=count, first=first)
        kind = "port"
        t_cfg = time.time() - t_a
        t_fwd = 0.0
    wall = time.time() - t0
    per_cfg = t_cfg / max(count, 1) + t_fwd / 64.0
    sample = (f"{count} of the 64 configurations (k1,k2)={w['pairs'][0]}, theta index {first}"
              f"{'..' + str(first + count - 1) if count > 1 else ''}, at {w['grid']}^3 plus the forward "
              f"transform amortised over 64; reference C + FFT shim (FFTW not installed; the shim stands "
              f"in for FFTW), shim FFT on {cores} thread{'s' if cores > 1 else ''}, estimator loops "
              f"single-threaded as in the reference; t_forward={t_fwd:.2f}s t_configs={t_cfg:.2f}s")
    return 1.0 / per_cfg, kind, cores, sample, wall, r


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU implementation (rank 0 only)."""
    if rank != 0:
        return
    w = workload(args.grid)
    dens, xhii = make_inputs(w)
    # CPU work has no warm-up effects; one configuration per step (~20-40 s
    # at 512^3), at most 3 timed steps so the run ends within a few minutes.
    steps = max(1, min(args.steps, 3))
    vals = []
    info = None
    t_all = time.time()
    for s in range(steps):
        v, kind, cores, sample, wall, _ = cpu_reference_sample(w, dens, xhii, first=s, count=1)
        vals.append(1.0 / v)
        info = (kind, cores, sample)
    per_cfg = float(np.mean(vals))
    value = 1.0 / per_cfg
    kind, cores, sample = info
    out = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=steps,
               warmup=0, requested_steps=args.steps, requested_warmup=args.warmup,
               ms_per_step=per_cfg * 1e3, higher_is_better=True, scaling="weak",
               vs_baseline=None, dtype="f64", data="synthetic", impl="reference",
               config=dict(workload=w["workload"], grid=w["grid"], box=w["box"],
                           binning="DERIVED", use_only_phase=1, configs_per_sweep=64),
               cpu_baseline=dict(value=value, unit=UNIT, cores=cores, kind=kind,
                                 sample=f"per step: {sample}"),
               e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0),
               wall_s=time.time() - t_all)
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------- GPU
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import polyspectrum_b200 as ps

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = workload(args.grid)
    dens_np, xhii_np = make_inputs(w)
    N, box = w["grid"], w["box"]
    sharded = world > 1 and not args.replicas
    if sharded:
        # weak scaling of the sharded path: 64 configurations per rank, whole
        # sweeps partitioned over the ranks, one all-gather of results per step
        from polyspectrum_b200 import multi
        all_cfgs = make_cfgs(ps, w, copies=world)
        parts = multi.partition(all_cfgs, world)
        cfgs = multi.share(all_cfgs, parts[rank])
        ncfg_total = len(all_cfgs)
        share_max = max(len(p) for p in parts)
    else:
        cfgs = make_cfgs(ps, w)
        ncfg_total = world * len(cfgs)
    ncfg = len(cfgs)

    # one non-default stream for torch and the library, so the timing events
    # (and torch's own work) are ordered with the library's kernels
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = ps.Context(N, box, methods=ps.PS_FP32_BATCHED, device=local_rank)
    ctx.set_stream(stream.cuda_stream)
    dens = torch.from_numpy(dens_np).to(dev)
    xhii = torch.from_numpy(xhii_np).to(dev)
    # the 64 configurations planned once (transform size of each pair group
    # autotuned at planning); executions replay one CUDA graph
    if args.tune_table:  # sub-grids fixed by an earlier run's table (profiling runs)
        with open(args.tune_table) as f:
            ctx.tune_import(f.read())
    plan = ctx.plan(cfgs, method=ps.PS_FP32_BATCHED, graph=True,
                    autotune=not (args.no_autotune or args.tune_table))
    tune_table = ctx.tune_export()
    if args.save_tune and rank == 0:
        with open(args.save_tune, "w") as f:
            f.write(tune_table)
    # the field spectrum is computed up to the band the plan's shells reach
    # (every mode the 64 configurations read; results identical to a full load)
    spectrum_band = plan.band if not args.full_spectrum else -1
    ctx.set_spectrum_band(spectrum_band)

    if sharded:
        resbuf = torch.zeros(8 * share_max, dtype=torch.float64, device=dev)
        gathered = torch.zeros(world * 8 * share_max, dtype=torch.float64, device=dev)

    def exchange():
        """The step's result exchange (sharded runs): this rank's results
        copied on the device, one NCCL all-gather over the ranks."""
        if sharded:
            plan.results_to_device(resbuf.data_ptr())
            dist.all_gather_into_tensor(gathered, resbuf)

    def step():
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
        r = plan.execute()
        exchange()
        return r

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_device(k, a, b):
        """Device time of k steps (plan prepare + field load + plan execution,
        results left on the device): the stream is held for ~50 ms first so the host queues
        all k steps before the first one starts, and no host work sits
        between the two events."""
        barrier()
        torch.cuda.synchronize()
        torch.cuda._sleep(100_000_000)  # about 50 ms at the B200's clock
        e0.record(stream)
        for _ in range(k):
            plan.prepare()  # DERIVED chain and exact counts, beside the field load
            ctx.set_field_async(ps.PS_FIELD_XHI_DENS, a, b, use_only_phase=1)
            plan.launch()
            exchange()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.synchronize()
        return max_over_ranks(e0.elapsed_time(e1))

    def steps_queued(k, a, b):
        """k steps queued without host waits: field load + plan execution each,
        results read back by the library in stream order."""
        subs = []
        for _ in range(k):
            plan.prepare()
            ctx.set_field_async(ps.PS_FIELD_XHI_DENS, a, b, use_only_phase=1)
            subs.append(plan.submit())
            exchange()
        ctx.synchronize()
        return subs

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(max(args.warmup, 3)):
        res = step()
    B32, N32 = res[0].copy(), res[1].copy()
    # then at least one second of the same work, so that the timed steps start
    # on a GPU at its steady clocks and power state
    t_warm = time.perf_counter()
    while time.perf_counter() - t_warm < 1.0:
        steps_queued(8, dens, xhii)

    # ---- timed region (inputs resident in HBM, larger than L2: no flush needed)
    clocks = ClockSampler(gpu_index(local_rank))
    clocks.wait_ready()
    barrier()
    torch.cuda.synchronize()
    t_clk0 = time.time()
    n_launch0 = ctx.launch_count()
    ms = timed_device(args.steps, dens, xhii)
    barrier()
    t_clk1 = time.time()
    timed_launches = ctx.launch_count() - n_launch0
    ms_step = ms / args.steps
    value = ncfg_total / (ms_step / 1e3)
    Bl, Nl, _, _ = plan.results()
    assert np.array_equal(Bl, B32) and np.array_equal(Nl, N32)

    # the same steps with the field transformed up to Nyquist (reported beside)
    value_full = None
    if spectrum_band >= 0:
        ctx.set_spectrum_band(-1)
        steps_queued(2, dens, xhii)
        value_full = ncfg_total / (timed_device(args.steps, dens, xhii) / args.steps / 1e3)
        Bl, Nl, _, _ = plan.results()
        assert np.array_equal(Bl, B32) and np.array_equal(Nl, N32)
        ctx.set_spectrum_band(spectrum_band)

    # ---- per-kernel roofline over a second pass of the same steps, events per launch
    ctx.set_profiling(True)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    stats = ctx.kernel_stats()
    ctx.set_profiling(False)
    peak, peak_kind = measured_peak()
    # the dominant HBM-bound kernel instance; the exact polygon counts
    # (pair_counts: integer histograms in shared memory, a few MB of mode
    # lists read) have no HBM roofline and are reported in `kernels` only
    hbm_stats = [s for s in stats if not s["name"].startswith("pair_counts")]
    dom = max(hbm_stats, key=lambda s: s["ms"]) if hbm_stats else None
    total_ms = sum(s["ms"] for s in stats) or 1.0
    roof = None
    if dom:
        achieved = dom["bytes"] / (dom["ms"] / 1e3) / 1e9
        # DRAM bytes per launch of this kernel instance from an ncu capture of the
        # same workload (profiles/dram_traffic.json), when one was taken
        traffic = None
        try:
            with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
                tr = json.load(f)
            if tr.get("workload") == w["workload"]:
                traffic = tr["kernels"].get(dom["name"], {}).get("dram_bytes_per_launch")
        except Exception:
            pass
        roof = dict(bound="hbm", kernel=dom["name"], achieved=achieved, peak=peak,
                    peak_source=peak_kind, unit="GB/s", frac=achieved / peak,
                    traffic=traffic, alg_bytes_per_launch=dom["bytes"] / dom["launches"],
                    avg_launch_ms=dom["ms"] / dom["launches"], launches=dom["launches"],
                    share_of_kernel_time=dom["ms"] / total_ms)
    all_alg = sum(s["bytes"] for s in stats)
    kernels = {s["name"]: dict(launches=s["launches"] // args.steps,
                               ms_per_step=s["ms"] / args.steps,
                               GBps=(s["bytes"] / (s["ms"] / 1e3) / 1e9) if s["ms"] > 0 and s["bytes"] > 0 else None)
               for s in stats}

    # ---- condition numbers of the configurations (one eager execution with
    # the |term| sums; the error of each B is about kappa * 2^-24)
    kplan = ctx.plan(cfgs, method=ps.PS_FP32_BATCHED, graph=False, kappa=True)
    ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
    _, _, kappa, cfg_out = kplan.execute()
    kplan.close()
    kmin32 = np.array([[cfg_out[q].kmin[j] for j in range(3)] for q in range(ncfg)])
    kmax32 = np.array([[cfg_out[q].kmax[j] for j in range(3)] for q in range(ncfg)])

    # ---- end to end: pinned host inputs, copies and result read-back inside.
    # Pipelined (the API's asynchronous calls): the upload of step k+1 runs on
    # the copy engine while step k's configurations run.  Serial: blocking
    # calls.  Each mode is timed three times, alternating.
    dens_h = torch.from_numpy(dens_np).pin_memory()
    xhii_h = torch.from_numpy(xhii_np).pin_memory()

    windows = [(t_clk0, t_clk1)]

    def timed_host(fn):
        barrier()
        torch.cuda.synchronize()
        w0 = time.time()
        t0 = time.perf_counter()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t0
        windows.append((w0, time.time()))
        return max_over_ranks(max(e0.elapsed_time(e1), t_wall * 1e3))

    def serial():
        for _ in range(args.steps):
            ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens_h, xhii_h, use_only_phase=1)
            plan.execute()
            exchange()

    load_stats = []

    def pipelined():
        steps_queued(args.steps, dens_h, xhii_h)
        load_stats.append(ctx.load_stats())

    steps_queued(2, dens_h, xhii_h)
    ms_pipe, ms_serial = [], []
    for _ in range(3):
        ms_pipe.append(timed_host(pipelined) / args.steps)
        ms_serial.append(timed_host(serial) / args.steps)
    ms_e2e = float(np.median(ms_pipe))
    e2e_value = ncfg_total / (ms_e2e / 1e3)
    ms_e2e_serial = float(np.median(ms_serial))
    time.sleep(0.1)
    clk = clocks.summary(windows)  # the device-timed and the end-to-end timed regions
    clocks.close()
    h2d = ctx.upload_bytes()  # the library composes dens*(1-xHII) on the host: one float grid per step
    d2h = ncfg * 8 * 8 + 4  # per configuration B, Npoly, 6 derived k bounds; one status word
    ls = load_stats[-1]
    host_load = dict(rows=ls["rows"], rows_raw=ls["rows_raw"], raw_frac=ls["rows_raw"] / max(ls["rows"], 1),
                     compose_ms=ls["compose_s"] * 1e3, raw_copy_ms=ls["raw_copy_ms"],
                     host_threads=ls["host_threads"], cpus=os.cpu_count(),
                     note="last load of the last pipelined repeat: rows sent raw (dens and xHII) vs composed "
                          "on host threads (one float per cell), host compose time and raw-row copy time")

    # ---- plain FP64 method on all 64 configurations (rank 0): the metric's
    # denominator and the error of every batched B against it
    plain = None
    parity = None
    if rank == 0 and world == 1 and not args.no_plain:
        plan.close()
        ctx.close()
        torch.cuda.empty_cache()
        with ps.Context(N, box, methods=ps.PS_FP64_PLAIN, device=local_rank) as c64:
            c64.set_stream(stream.cuda_stream)
            c64.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
            c64.batch(cfgs[:1], ps.PS_FP64_PLAIN)
            torch.cuda.synchronize()
            e0.record(stream)
            c64.get_FT_field(ps.PS_FIELD_XHI_DENS, dens, xhii, use_only_phase=1)
            e1.record(stream)
            torch.cuda.synchronize()
            t_fwd64 = e0.elapsed_time(e1)
            e0.record(stream)
            B64, N64, _, out64 = c64.batch(cfgs, ps.PS_FP64_PLAIN)
            e1.record(stream)
            torch.cuda.synchronize()
            t_cfg64 = e0.elapsed_time(e1) / ncfg
        per_cfg64 = t_cfg64 + t_fwd64 / ncfg
        rel = np.abs(B32 - B64) / np.abs(B64)
        kmin64 = np.array([[out64[q].kmin[j] for j in range(3)] for q in range(ncfg)])
        kmax64 = np.array([[out64[q].kmax[j] for j in range(3)] for q in range(ncfg)])
        plain = dict(configs_per_s=1e3 / per_cfg64, ms_per_config=t_cfg64, forward_ms=t_fwd64,
                     sample=f"all {ncfg} configurations of the sweep",
                     batched_vs_plain_speedup=value / world / (1e3 / per_cfg64),
                     max_rel_err_B_fp32_vs_fp64=float(rel.max()),
                     counts_equal=bool(np.array_equal(N32, np.rint(N64))))
        eps32 = 2.0 ** -24
        parity = dict(
            tolerance="|dB| <= 1e-5 |B| per configuration (no absolute floor); counts exact; DERIVED k-ranges "
                      "bit-identical",
            fp64_plain=dict(configs=ncfg, max_rel_err_B=float(rel.max()), median_rel_err_B=float(np.median(rel)),
                            within_1e_5=bool((rel <= 1e-5).all()),
                            counts_equal=bool(np.array_equal(N32, np.rint(N64))),
                            derived_equal=bool(np.array_equal(kmin32, kmin64) and np.array_equal(kmax32, kmax64))),
            kappa=dict(max=float(np.max(kappa)), median=float(np.median(kappa)),
                       at_max_rel_err=float(kappa[int(np.argmax(rel))]),
                       max_rel_err_over_kappa_eps32=float(np.max(rel / (kappa * eps32)))))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference itself on configuration 0 of the sweep ((k1,k2) = (0.2,0.5),
        # theta index 0) at 512^3, all host threads; its result checks the GPU's
        v, kind, cores, sample, wall, r = cpu_reference_sample(w, dens_np, xhii_np)
        cpu = dict(value=v, unit=UNIT, cores=cores, kind=kind, sample=sample, nproc=os.cpu_count(),
                   cpu_model=cpu_model(),
                   note="the reference's C with this repository's FP64 FFT shim standing in for FFTW (not "
                        "installed); the reference's MPI path is unavailable on this box (no MPI / FFTW-MPI)")
        if parity is not None:
            rel0 = abs(B32[0] - r.B[0]) / abs(r.B[0])
            parity["reference"] = dict(
                config="(k1,k2)=(0.2,0.5) h/Mpc, theta index 0, 512^3 (pair group on the 128-point sub-grid)",
                kind=kind, B_reference=float(r.B[0]), B_gpu=float(B32[0]), rel_err_B=float(rel0),
                within_1e_5=bool(rel0 <= 1e-5), npoly_reference=float(r.npoly[0]), npoly_gpu=float(N32[0]),
                npoly_equal=bool(N32[0] == np.rint(r.npoly[0])),
                derived_equal=bool(np.array_equal(kmin32[0], r.kmin[0]) and np.array_equal(kmax32[0], r.kmax[0])))
        if not args.no_serial_cpu:
            # one thread (the reference's serial path) at sizes where that is cheap
            serial_runs = []
            for g in (128, 256):
                ws = workload(g)
                ds, xs = make_inputs(ws)
                vs, kind_s, _, sample_s, _, _ = cpu_reference_sample(ws, ds, xs, threads=1)
                serial_runs.append(dict(grid=g, value=vs, unit=UNIT, cores=1, kind=kind_s, sample=sample_s))
            cpu["serial_1_thread"] = serial_runs

    if rank == 0:
        out = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps,
                   warmup=max(args.warmup, 3), ms_per_step=ms_step, higher_is_better=True,
                   scaling="weak", vs_baseline=None, dtype="f32 (FP64 counts and sums)",
                   data="synthetic (seeded XHI_DENS field: 32000 spheres x lognormal density)",
                   config=dict(workload=w["workload"], grid=N, box=box, pairs=w["pairs"],
                               theta_bins=w["num_values"], configs_per_step=ncfg,
                               binning="DERIVED", kbinwidth=1.0, use_only_phase=1,
                               l2="inputs (2 x 512 MiB) and every pass larger than L2; no flush",
                               parallelism=("single GPU" if world == 1 else
                                            f"replicas x{world}" if not sharded else
                                            f"sharded over {world} ranks: {ncfg_total} configurations "
                                            f"(64 per rank, whole sweeps per rank), one NCCL all-gather "
                                            f"of the results per step"),
                               configs_total=ncfg_total,
                               subgrids=[int(ln.split()[-1]) for ln in tune_table.splitlines() if ln.startswith("grid")],
                               tune_table=[ln for ln in tune_table.splitlines() if ln.strip()],
                               spectrum_band=spectrum_band, value_full_spectrum=value_full),
                   e2e=dict(value=e2e_value, unit=UNIT, h2d_bytes_per_step=h2d,
                            d2h_bytes_per_step=d2h, ms_per_step=ms_e2e,
                            ms_per_step_repeats=ms_pipe,
                            mode="pipelined: ps_gpu_plan_prepare + ps_gpu_set_field_async + ps_gpu_plan_submit per step, "
                                 "one ps_gpu_synchronize after the last; the library composes "
                                 "dens*(1-xHII) of the two host grids on host threads and uploads one",
                            serial_value=ncfg_total / (ms_e2e_serial / 1e3),
                            serial_ms_per_step=ms_e2e_serial, serial_ms_per_step_repeats=ms_serial,
                            serial_mode="ps_gpu_set_field + ps_gpu_plan_execute per step (blocking)",
                            host_load=host_load),
                   gpu_launches=timed_launches, roofline=roof,
                   whole_step=dict(alg_bytes=all_alg / args.steps,
                                   achieved_GBps=all_alg / args.steps / (ms_step / 1e3) / 1e9,
                                   frac=all_alg / args.steps / (ms_step / 1e3) / 1e9 / peak,
                                   peak=peak, peak_source=peak_kind),
                   kernels=kernels, clocks=clk, plain_fp64=plain, parity=parity, cpu_baseline=cpu)
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=512, help="grid size (the workload is 512)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-serial-cpu", action="store_true",
                    help="skip the 1-thread reference runs at 128^3 and 256^3")
    ap.add_argument("--replicas", action="store_true",
                    help="with --gpus N > 1: N independent replicas of the 64-configuration step instead of the "
                         "sharded path")
    ap.add_argument("--full-spectrum", action="store_true",
                    help="transform the field up to Nyquist instead of the plan's band")
    ap.add_argument("--no-autotune", action="store_true",
                    help="smallest alias-free sub-grid per pair group, no timing at planning")
    ap.add_argument("--save-tune", default=None, help="write the plan's sub-grid table to this file")
    ap.add_argument("--tune-table", default=None,
                    help="take the sub-grids from a table written by --save-tune (no autotuning)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
