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


# ---------------------------------------------------------------------------
# coil-sharded CG-SENSE (mirt_b200.sharded) on CPU ranks with the FP64 oracle
# operator standing in for the device NUFFT
# ---------------------------------------------------------------------------
def _sense_case():
    """A small SENSE problem (N = 24, K = 48, 4 coils, radial, Reg1 beta)."""
    sys.path.insert(0, ROOT)
    from mirt_b200 import workloads as wl
    rng = np.random.default_rng(77)
    N, C = 24, 4
    om = wl.ga_radial(20, 2 * N, start=0.3)
    sens = wl.coil_maps((N, N), C, rng).transpose(1, 0, 2).astype(np.complex128)
    xt = wl.ellipses(N, 5, rng).T
    return N, om, sens, xt


class _TorchOp:
    """oracle Sense64 (FP64 numpy) behind the torch interface of the sharded solver."""

    def __init__(self, S):
        self.S = S

    def forward(self, x):
        import torch
        return torch.from_numpy(self.S.forward(x.numpy()))

    def adjoint(self, r):
        import torch
        return torch.from_numpy(self.S.adjoint(r.numpy()))

    def reg(self, x):
        import torch
        return torch.from_numpy(self.S.reg(x.numpy()))


def _sharded_iterates(coils, niter):
    import torch
    from mirt_b200.sharded import qpwls_pcg1_coil_sharded
    from oracle import sense_ref as sr
    N, om, sens, xt = _sense_case()
    full = sr.Sense64(om, N, 2 * N, sens, beta=0.0)
    y = full.forward(xt)                               # data of every coil
    beta = 2.0 ** -8 * len(om) * np.mean(np.sum(np.abs(sens) ** 2, axis=-1))
    S = sr.Sense64(om, N, 2 * N, sens[:, :, coils], beta)
    x0 = torch.zeros((N, N), dtype=torch.complex128)
    xs = qpwls_pcg1_coil_sharded(x0, _TorchOp(S), torch.from_numpy(y[:, coils]), niter,
                                 iterates=True)
    return np.stack([x.numpy() for x in xs]), full, y, beta


def _sharded_worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    xs, _, _, _ = _sharded_iterates(list(range(rank, 4, world)), 6)
    q.put((rank, xs))
    dist.barrier()
    dist.destroy_process_group()


def test_coil_sharded_cg_sense_two_ranks_equals_one():
    """Two gloo ranks, coils {0, 2} and {1, 3}: every iterate of the sharded
    qpwls_pcg1 equals the one-rank iterate to FP64 rounding (the ranks agree
    with each other exactly), and the one-rank iterates follow the oracle's
    qpwls_pcg1 (wls/qpwls_pcg1.m:94-189), whose gradient is recomputed from
    A x instead of carried along."""
    import torch.multiprocessing as mp
    from oracle import sense_ref as sr
    one, full, y, beta = _sharded_iterates([0, 1, 2, 3], 6)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(out[0], out[1])
    scale = np.abs(one[-1]).max()
    assert np.abs(out[0] - one).max() <= 1e-12 * scale
    N = one.shape[-1]
    ref = sr.qpwls_pcg1(np.zeros((N, N)), sr.Sense64(full.st["om"], N, 2 * N, full.sens, beta),
                        None, y, 6)
    assert np.abs(one - np.stack(ref)).max() <= 1e-9 * scale
