"""The multi-GPU path of bench.py is replicas: each rank images its own clips,
the only collectives are a barrier and the max of the timings.  Checked here
with world_size 2 on CPU (gloo)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = 100.0 + 50.0 * rank          # rank 1 is the slowest
    ms = bench.max_over_ranks_on(local_ms, world, torch.device("cpu"))
    dist.barrier()
    out[rank] = (ms, bench.whole_job_rate(4, world, ms), tuple(bench.rank_seeds(rank, 4)))
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 150.0                    # max over ranks
    assert out[0][1] == pytest.approx(8 / 0.150)              # all ranks' clips / slowest time
    assert not set(out[0][2]) & set(out[1][2])                 # disjoint clips per rank
