"""Multi-rank host logic of bench.py on the CPU (gloo, world size 2).

The batched NUFFT shards without exchange: each rank runs its own seeded
batch of slices, and only the timing is combined -- the job time is the
slowest rank's, the units are the sum over ranks.  The reference arm runs on
rank 0 only; the other ranks exit without work.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    t, u = bench.combine_over_ranks(1.0 + rank, 10.0 * (rank + 1), world, "cpu")
    om, moff = bench.rank_batch(bench.WORKLOADS["c1"], rank)
    q.put((rank, t, u, float(om.sum()), len(moff)))
    dist.barrier()
    dist.destroy_process_group()


def test_combine_and_independent_batches_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, t, u, _, _ in out:
        assert t == 2.0 and u == 30.0          # max of times, sum of units
    assert out[0][3] != out[1][3]               # each rank its own trajectories


def test_reference_arm_other_ranks_do_no_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        steps, warmup, workload, gpus = 1, 1, "c1", 2
    assert bench.run_reference(A(), bench.WORKLOADS["c1"]) == 0
