"""Multi-rank plumbing of the benchmark on CPU (two gloo ranks): every rank runs its own replica, the job's
time is the slowest rank's, and the throughput counts the units of all ranks. No GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    ms_local = 10.0 * (rank + 1)                     # rank 1 is the slow one
    ms = bench.max_over_ranks(ms_local, dist)
    out[rank] = (ms, bench.job_rate(1000, 5, world, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0][0] == out[1][0] == 20.0
    assert out[0][1] == pytest.approx(1000 * 5 * 2 / 0.020)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_rate(10, 2, 1, 1000.0) == pytest.approx(20.0)
