"""The replica form of bench.py across ranks, on the CPU with the gloo backend (world size 2):
every rank times its own replica, the job time is the maximum over ranks and the job value counts
every rank's steps."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dev_ms, wall = bench.max_over_ranks([100.0 + 50.0 * rank, 2.0 - rank], world, "cpu")
        out[rank] = (dev_ms, wall, bench.job_throughput(3, world, dev_ms / 1e3))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_value():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, 29513, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        for r in range(2):
            dev_ms, wall, value = out[r]
            assert dev_ms == 150.0 and wall == 2.0
            assert value == pytest.approx(6 / 0.150)
