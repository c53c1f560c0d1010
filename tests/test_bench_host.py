"""bench.py's multi-rank arithmetic: the job time is the slowest rank's and
the value is the units all ranks processed over it (two gloo ranks on CPU)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 10.0 * (rank + 1)
    t = bench.max_over_ranks(dist, ms)
    q.put((rank, t, bench.job_rate(1000, world, t)))
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    for rank, t, v in res:
        assert t == 20.0 and v == pytest.approx(1000 * 2 / 0.020)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(None, 3.5) == 3.5
