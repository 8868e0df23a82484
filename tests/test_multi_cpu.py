"""Configuration sharding over ranks (polyspectrum_b200/multi.py) on the CPU:
the partition keeps theta sweeps together and covers every configuration
once; world-size 2 and 3 gloo process groups (127.0.0.1) gather the result of
a deterministic stand-in evaluation back into the caller's order; a rank that
fails makes every rank raise instead of leaving the others waiting."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ps():
    import polyspectrum_b200 as ps
    from polyspectrum_b200 import build
    build.build(quiet=True)
    ps.lib()
    return ps


def bench_like_cfgs(ps):
    out = []
    for k1, k2 in ((0.2, 0.5), (0.5, 0.8), (0.8, 1.2), (1.0, 1.5)):
        c, _, _ = ps.read_params_to_kvectors(512, 400.0, 3, k1=k1, k2=k2, num_values=16, kbinningCase=1)
        out += [c[i] for i in range(len(c))]
    eq, _, _ = ps.read_params_to_kvectors(512, 400.0, 3, equilateral=1, num_values=5)
    p2, _, _ = ps.read_params_to_kvectors(512, 400.0, 2, num_values=2)
    out += [eq[i] for i in range(len(eq))] + [p2[i] for i in range(len(p2))]
    return out


def fake_evaluate(sub):
    """Deterministic stand-in for ctx.batch: values from the configuration."""
    n = len(sub)
    B = np.array([sum(sub[i].k[l] for l in range(sub[i].n)) * 1.5 for i in range(n)])
    Np = np.array([float(sub[i].n * 10 + int(round(sub[i].k[sub[i].n - 1] * 1000)) % 7) for i in range(n)])
    for i in range(n):
        for l in range(sub[i].n):
            sub[i].kmin[l] = sub[i].k[l] - 0.01
            sub[i].kmax[l] = sub[i].k[l] + 0.01
    return B, Np, sub


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition(ps, world):
    from polyspectrum_b200.multi import group_key, partition
    cfgs = bench_like_cfgs(ps)
    parts = partition(cfgs, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(cfgs)))
    owner = {i: r for r, p in enumerate(parts) for i in p}
    keys = {}
    for i in range(len(cfgs)):
        keys.setdefault(group_key(cfgs[i], i), set()).add(owner[i])
    assert all(len(v) == 1 for v in keys.values())  # no group split
    if world <= 4:
        assert all(len(p) > 0 for p in parts)
    assert partition(cfgs, world) == parts  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir, fail_rank):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    import polyspectrum_b200 as ps
    from polyspectrum_b200.multi import ShardError, evaluate_sharded
    from test_multi_cpu import bench_like_cfgs, fake_evaluate
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfgs = bench_like_cfgs(ps)

        def ev(sub):
            if rank == fail_rank:
                raise RuntimeError("planted failure")
            return fake_evaluate(sub)
        try:
            res = evaluate_sharded(None, cfgs, evaluate=ev)
            np.savez(os.path.join(outdir, f"r{rank}.npz"), B=res.B, npoly=res.npoly, kmin=res.kmin, kmax=res.kmax)
        except ShardError as e:
            with open(os.path.join(outdir, f"r{rank}.err"), "w") as f:
                f.write(str(e))
    finally:
        dist.destroy_process_group()


def _spawn(world, tmp_path, fail_rank=-1):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path), fail_rank), nprocs=world, join=True)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_gather_matches_serial(ps, tmp_path, world):
    from polyspectrum_b200.multi import evaluate_sharded
    cfgs = bench_like_cfgs(ps)
    serial = evaluate_sharded(None, cfgs, evaluate=fake_evaluate)
    _spawn(world, tmp_path)
    for r in range(world):
        got = np.load(os.path.join(str(tmp_path), f"r{r}.npz"))
        np.testing.assert_array_equal(got["B"], serial.B)
        np.testing.assert_array_equal(got["npoly"], serial.npoly)
        np.testing.assert_array_equal(got["kmin"], serial.kmin)
        np.testing.assert_array_equal(got["kmax"], serial.kmax)
    # the stand-in is per-configuration, so the serial result is the direct one
    B, Np, _ = fake_evaluate(cfgs)
    np.testing.assert_array_equal(serial.B, B)


def test_failing_rank_raises_everywhere(ps, tmp_path):
    _spawn(2, tmp_path, fail_rank=1)
    for r in range(2):
        msg = open(os.path.join(str(tmp_path), f"r{r}.err")).read()
        assert "fail" in msg
    assert "planted failure" in open(os.path.join(str(tmp_path), "r1.err")).read()


class FakePlan:
    """Stand-in for a ps.Plan of a share: launch() computes, results() returns."""

    def __init__(self, sub, fail=False):
        self.sub = sub
        self.fail = fail
        self.res = None

    def launch(self):
        if self.fail:
            raise RuntimeError("planted launch failure")
        self.res = fake_evaluate(self.sub)

    def results(self):
        B, Np, out = self.res
        return B, Np, None, out

    def close(self):
        pass


def _plan_worker(rank, world, port, outdir, fail_rank):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    import polyspectrum_b200 as ps
    from polyspectrum_b200.multi import ShardError, ShardedPlan
    from test_multi_cpu import FakePlan, bench_like_cfgs
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfgs = bench_like_cfgs(ps)
        sp = ShardedPlan(None, cfgs, make_plan=lambda sub: FakePlan(sub, fail=rank == fail_rank))
        try:
            for _ in range(2):  # two steps, the same collective sequence on every rank
                res = sp.execute()
            np.savez(os.path.join(outdir, f"r{rank}.npz"), B=res.B, npoly=res.npoly, kmin=res.kmin, kmax=res.kmax)
        except ShardError as e:
            with open(os.path.join(outdir, f"r{rank}.err"), "w") as f:
                f.write(str(e))
        sp.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,fail_rank", [(2, -1), (3, -1), (2, 0)])
def test_sharded_plan_steps(ps, tmp_path, world, fail_rank):
    """ShardedPlan: each rank plans its share once, every step gathers all
    results in the caller's order; a rank whose launch fails makes every rank
    raise at the same step."""
    import torch.multiprocessing as mp

    from polyspectrum_b200.multi import evaluate_sharded
    cfgs = bench_like_cfgs(ps)
    serial = evaluate_sharded(None, cfgs, evaluate=fake_evaluate)
    mp.spawn(_plan_worker, args=(world, _free_port(), str(tmp_path), fail_rank), nprocs=world, join=True)
    for r in range(world):
        if fail_rank >= 0:
            msg = open(os.path.join(str(tmp_path), f"r{r}.err")).read()
            assert "fail" in msg
            continue
        got = np.load(os.path.join(str(tmp_path), f"r{r}.npz"))
        np.testing.assert_array_equal(got["B"], serial.B)
        np.testing.assert_array_equal(got["npoly"], serial.npoly)
        np.testing.assert_array_equal(got["kmin"], serial.kmin)
