"""GPU: a captured batched NUFFT step (mirt_nufft_capture) replays the eager
forward + adjoint exactly (every kernel is deterministic), twice in a row and
after the input changed in place."""
from __future__ import annotations

import numpy as np
import pytest

import mirt_b200 as mb
from mirt_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("C", [8, 32])
def test_graph_replay_matches_eager(C):
    """C = 32: the captured step holds the TMA-staged gather (its tensor map a
    by-value kernel parameter) and the row sweep with its ordering pass."""
    import torch
    rng = np.random.default_rng(11)
    om, moff, _ = wl.batch_ga_radial(3, 20, 40, 128, rng)
    G = mb.NufftPlan(om, (64, 64), (6, 6), (128, 128), n_shift=(32, 32), Ld=1024, ncol=C,
                     slice_moff=moff)
    if C == 32:
        cfg = G.config()
        assert cfg["gather_tma"] in (1, 2) and cfg["spread_sweep"] != 0
    x = torch.randn(G.image_shape, dtype=torch.complex64, device="cuda")
    X = torch.empty(G.sample_shape, dtype=torch.complex64, device="cuda")
    xa = torch.empty(G.image_shape, dtype=torch.complex64, device="cuda")
    Xe = G.forward(x)
    xe = G.adjoint(Xe)
    g = G.capture(x, X, xa)
    for _ in range(2):
        g.launch()
        torch.cuda.synchronize()
        assert torch.equal(X, Xe) and torch.equal(xa, xe)
    x.mul_(2.0)
    g.launch()
    torch.cuda.synchronize()
    assert torch.equal(X, G.forward(x)) and torch.equal(xa, G.adjoint(X))
    g.close()
