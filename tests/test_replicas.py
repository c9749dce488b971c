"""The multi-GPU form of the benchmark is replicas: each rank steps its own copy of the grid, and
the job's time is the slowest rank's. Its reduction is checked here on CPU ranks (gloo, two
processes): every rank reports the maximum, and the rate counts every rank's cells."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, times, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    ms, value = bench.aggregate(times[rank], 100, 1_000_000, dist, "cpu")
    out[rank] = (ms, value)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_slowest_rank_sets_the_time(world):
    times = [3.0, 5.0]
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=rank_main, args=(r, world, free_port_cached[0], times, out))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        ms, value = out[r]
        assert ms == 5.0
        assert value == pytest.approx(world * 100 * 1_000_000 / 5e-3 / 1e9)


def test_one_rank_without_a_group():
    import bench
    assert bench.aggregate(2.0, 10, 1000) == (2.0, 10 * 1000 / 2e-3 / 1e9)


free_port_cached = [free_port()]
