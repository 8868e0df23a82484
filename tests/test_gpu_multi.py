"""Configuration sharding through a real NCCL process group on the GPU: a
single-rank group (the GPU tests get one device) must gather exactly what a
direct batch returns, DERIVED write-back included."""
import datetime
import socket

import numpy as np
import pytest

from _cases import field_args, fields

pytestmark = pytest.mark.gpu


def test_sharded_single_rank_nccl(gpu_lib):
    import torch
    import torch.distributed as dist

    from polyspectrum_b200.multi import evaluate_sharded
    ps = gpu_lib
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        n_grid, box = 32, 200.0
        dd, xx = field_args(2, *fields(n_grid, box))
        cfgs = []
        for k1, k2 in ((0.1, 0.14), (0.12, 0.2)):
            c, _, _ = ps.read_params_to_kvectors(n_grid, box, 3, k1=k1, k2=k2, num_values=5, kbinningCase=1)
            cfgs += [c[i] for i in range(len(c))]
        with ps.Context(n_grid, box) as ctx:
            ctx.get_FT_field(2, dd, xx, use_only_phase=1)
            res = evaluate_sharded(ctx, cfgs)
            B, Np, _, out = ctx.batch(cfgs, ps.PS_FP32_BATCHED)
        np.testing.assert_array_equal(res.B, B)
        np.testing.assert_array_equal(res.npoly, Np)
        for i in range(len(cfgs)):
            np.testing.assert_array_equal(res.kmin[i], list(out[i].kmin))
            np.testing.assert_array_equal(res.kmax[i], list(out[i].kmax))
    finally:
        dist.destroy_process_group()
