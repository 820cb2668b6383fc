"""The N > 1 path of bench.py (independent replicas, one per rank): the
job's time is the slowest rank's and the throughput sums the replicas.
Two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import REPO


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, REPO)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, dist, "cpu")
        out[rank] = (ms_max, bench.replica_mlups(world, 1000, 100, ms_max))
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    import random

    world = 2
    port = random.randint(20000, 40000)
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms_max, mlups = res[0]
    assert ms_max == 15.0
    assert mlups == pytest.approx(2 * 1000 * 100 / 15e-3 / 1e6)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, REPO)
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
