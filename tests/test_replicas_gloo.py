"""The multi-rank bench logic on CPU: two gloo ranks, each timing its own
replica; the job's time is the slowest rank's and the rate counts the units
of every rank (weak scaling).  No GPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 10 * (r + 1) ms for 5 steps of 1000 units
        ms = 10.0 * (rank + 1)
        job_ms = bench.reduce_max(ms, dist, device="cpu")
        rate = bench.whole_job_rate(world, 1000, 5, job_ms)
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.replica_seed(rank))
        out[rank] = (job_ms, rate, seeds)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for rank in range(world):
        job_ms, rate, seeds = res[rank]
        assert job_ms == 20.0
        assert rate == pytest.approx(world * 1000 * 5 / 0.020)
        assert len(set(seeds)) == world  # independent replicas


def test_single_process_helpers():
    assert bench.reduce_max(3.5, None) == 3.5
    assert bench.whole_job_rate(1, 10, 2, 1000.0) == 20.0
