"""Configurations sharded over ranks, one process per GPU.

Given the field spectrum, the estimator's configurations are independent.
Each rank loads the field and runs the forward transform itself (the input
grids are replicated; exchanging the spectrum would move more bytes than the
transform costs), evaluates its share of the configurations, and one
all-gather per call hands every rank the whole result in the caller's order.
The reference distributes the other way round - slabs of one grid over MPI
ranks with an allreduce per grid sum (polyspectrum.c:144-153, :239-245) -
because its grids do not fit one node's memory; an N^3 = 1024^3 FP32 grid
fits one GPU here, so ranks split work, not grids.

Shares keep the configurations of one theta sweep together (they share legs 0
and 1, which the batched method transforms once per sweep) and are balanced
by an estimate of each group's transform volume.  Every rank takes the same
collective steps in the same order, error paths included: a rank whose
evaluation fails still joins the status exchange, and then every rank raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

PAYLOAD = 3 + 2 * 8  # index, B, Npoly, kmin[8], kmax[8]


class ShardError(RuntimeError):
    """A rank failed to evaluate its share (raised on every rank)."""


def group_key(cfg, index: int) -> tuple:
    """Configurations with equal keys go to the same rank: theta sweeps (n = 3,
    shared legs 0 and 1); n = 2 configurations in blocks of 16 (one k-space
    pass of the batched method); anything else alone."""
    if cfg.n == 3:
        return (3, cfg.kbinningCase, cfg.kbinwidth, cfg.k[0], cfg.k[1])
    if cfg.n == 2:
        return (2, index // 16)
    return (cfg.n, index)


def group_cost(cfgs, members) -> float:
    """Transform volume estimate: (sum of the leg lengths)^3 of the largest
    member (the alias-free grid of a pair group grows with it), plus a small
    per-configuration term for the dot passes."""
    big = max(sum(abs(cfgs[i].k[l]) for l in range(cfgs[i].n)) for i in members)
    return big ** 3 + 1e-3 * len(members) * big ** 3


def partition(cfgs, world: int) -> list[list[int]]:
    """Indices of the configurations each rank evaluates: whole groups,
    longest-processing-time first onto the least loaded rank (deterministic:
    ties go to the lower rank, groups in first-appearance order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    groups: dict[tuple, list[int]] = {}
    for i in range(len(cfgs)):
        groups.setdefault(group_key(cfgs[i], i), []).append(i)
    order = sorted(groups.values(), key=lambda m: (-group_cost(cfgs, m), m[0]))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for members in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].extend(members)
        load[r] += group_cost(cfgs, members)
    return [sorted(p) for p in parts]


@dataclass
class ShardedResult:
    B: np.ndarray
    npoly: np.ndarray
    kmin: np.ndarray  # [nconf, 8] k ranges after DERIVED write-back
    kmax: np.ndarray
    parts: list


def _dist():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist
    except Exception:
        pass
    return None


def _all_gather(dist, arr: np.ndarray) -> list[np.ndarray]:
    import torch
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [o.cpu().numpy() for o in out]


def _gather(dist, parts, rank, n, local, err):
    """Status exchange, then one all-gather of every rank's results, unpacked
    into the caller's order.  `local` = (B, Npoly, cfgs_out) of this rank's
    share or None; `err` = this rank's exception or None."""
    mine = parts[rank]
    payload = np.zeros((max(len(p) for p in parts) if parts else 0, PAYLOAD))
    status = 1 if err is not None else 0
    if err is None and mine:
        B, Np, out = local
        for j, i in enumerate(mine):
            payload[j, 0] = i
            payload[j, 1] = B[j]
            payload[j, 2] = Np[j]
            payload[j, 3:11] = list(out[j].kmin)
            payload[j, 11:19] = list(out[j].kmax)
    if dist:
        flags = _all_gather(dist, np.array([float(status)]))
        failed = [q for q, f in enumerate(flags) if f[0] != 0.0]
    else:
        failed = [0] if status else []
    if failed:
        if status:
            raise ShardError(f"rank {rank} failed: {err}") from err
        raise ShardError(f"ranks {failed} failed to evaluate their share")
    blocks = _all_gather(dist, payload) if dist else [payload]
    B = np.full(n, np.nan)
    Np = np.full(n, np.nan)
    kmin = np.zeros((n, 8))
    kmax = np.zeros((n, 8))
    for q, blk in enumerate(blocks):
        for j in range(len(parts[q])):
            i = int(blk[j, 0])
            B[i], Np[i] = blk[j, 1], blk[j, 2]
            kmin[i], kmax[i] = blk[j, 3:11], blk[j, 11:19]
    return ShardedResult(B, Np, kmin, kmax, parts)


def share(cfgs, mine):
    """The configurations of indices `mine` as a ps_cfg array."""
    from . import ps_cfg
    sub = (ps_cfg * max(len(mine), 1))()
    for j, i in enumerate(mine):
        C.memmove(C.byref(sub[j]), C.byref(cfgs[i]), C.sizeof(ps_cfg))
    return sub if mine else sub[:0]


def evaluate_sharded(ctx, cfgs, method: int | None = None, evaluate=None) -> ShardedResult:
    """Evaluate `cfgs` over all ranks of the default process group (or alone
    when none is initialised).  `evaluate(sub_cfgs) -> (B, Npoly, cfgs_out)`
    defaults to ctx.batch with `method` (PS_FP32_BATCHED)."""
    from . import PS_FP32_BATCHED
    dist = _dist()
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist else (0, 1)
    parts = partition(cfgs, world)
    mine = parts[rank]
    if evaluate is None:
        m = PS_FP32_BATCHED if method is None else method

        def evaluate(sub):
            B, Np, _, out = ctx.batch(sub, m)
            return B, Np, out
    local, err = None, None
    try:
        if mine:
            local = evaluate(share(cfgs, mine))
    except Exception as e:  # joins the status exchange, then raises everywhere
        err = e
    return _gather(dist, parts, rank, len(cfgs), local, err)


class ShardedPlan:
    """A configuration list split over the ranks of the default process group
    (whole theta sweeps, balanced as `partition` does), each rank holding one
    plan of its share (PS_FP32_BATCHED, CUDA graph, optionally autotuned).
    execute() runs this rank's plan on the field loaded last and returns every
    rank's results through one all-gather; launch() / gather() split that into
    the stream work and the exchange.  `make_plan(sub_cfgs)` replaces
    ctx.plan (tests)."""

    def __init__(self, ctx, cfgs, autotune: bool = True, graph: bool = True, make_plan=None):
        dist = _dist()
        self.dist = dist
        self.rank, self.world = (dist.get_rank(), dist.get_world_size()) if dist else (0, 1)
        self.n = len(cfgs)
        self.parts = partition(cfgs, self.world)
        self._err = None
        mine = self.parts[self.rank]
        self.plan = None
        err = None
        try:
            if mine:
                sub = share(cfgs, mine)
                self.plan = make_plan(sub) if make_plan else ctx.plan(sub, graph=graph, autotune=autotune)
        except Exception as e:
            err = e
        # every rank learns whether every plan was made
        mine_flag = np.array([float(err is not None)])
        flags = _all_gather(dist, mine_flag) if dist else [mine_flag]
        failed = [q for q, f in enumerate(flags) if f[0] != 0.0]
        if failed:
            if err is not None:
                raise ShardError(f"rank {self.rank} failed to plan its share: {err}") from err
            raise ShardError(f"ranks {failed} failed to plan their share")

    @property
    def band(self) -> int:
        """Largest |component| of a mode this rank's share reads (-1: no share)."""
        return self.plan.band if self.plan is not None else -1

    def launch(self):
        """Queue this rank's plan execution (results stay on the device).  A
        failure is kept and reported by the next gather(), on every rank."""
        try:
            if self.plan is not None:
                self.plan.launch()
        except Exception as e:
            self._err = e

    def gather(self) -> ShardedResult:
        """Results of the latest launch on every rank (waits; one all-gather)."""
        local, err = None, self._err
        self._err = None
        try:
            if err is None and self.plan is not None:
                B, Np, _, out = self.plan.results()
                local = (B, Np, out)
        except Exception as e:
            err = e
        return _gather(self.dist, self.parts, self.rank, self.n, local, err)

    def execute(self) -> ShardedResult:
        self.launch()
        return self.gather()

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None
