"""Multi-GPU runs are replicas: each rank runs its own seeded batch with no
data exchange, and the job time is the maximum over ranks. This checks that
logic with two gloo ranks on the CPU (no GPU involved)."""
import os
import socket

import numpy as np
import torch.multiprocessing as tmp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    import bench
    import multistageqw_b200 as M
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    t = 10.0 + 5.0 * rank  # this rank's step time
    worst = bench.max_over_ranks(t, world, dist, "cpu")
    seed = bench.replica_seed(20, rank)
    batch = M.sk_instances(12, 2, seed)
    out[rank] = (worst, seed, float(batch.sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    mgr = tmp.Manager()
    out = mgr.dict()
    tmp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 15.0          # max over ranks
    assert out[0][1] != out[1][1]                  # distinct seeds
    assert out[0][2] != out[1][2]                  # distinct batches


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_seed(20, 0) == 20
    assert np.isfinite(bench.replica_seed(20, 7))
