"""The multi-process path of bench.py on CPU: world_size 2 over gloo, one
replica per rank, the job time is the slowest rank's and the rate counts the
units of all ranks."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(dist, 1.0 + rank, "cpu")  # rank 1 is slower
        out[rank] = (t, bench.job_rate(world, 100.0, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 100.0)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(dist, 3.5, "cpu") == 3.5
    assert bench.job_rate(1, 10.0, 2.0) == 5.0
