"""Learned density compensation: the FP64 restatement of the network and the
features (CPU).  Pins the oracle itself: back-propagated gradients against
central finite differences, BF16 rounding against torch's, and the neighbour
histogram against a brute-force count."""
import numpy as np
import pytest

from oracle import mlp_ref


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 10000),
                        np.float32([0.0, -0.0, 1.0, 3.0e38, 1e-40])])
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(mlp_ref.bf16_round(x), ref)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = mlp_ref.init_params(rng)
    x = rng.standard_normal((37, mlp_ref.NFEAT))
    y = rng.standard_normal(37)
    loss, g = mlp_ref.grad(p, x, y)
    # differentiate the FP64 network at the BF16-rounded point directly
    pb = mlp_ref.bf16_round(p).astype(np.float64)

    def f(q):
        w = mlp_ref.unpack(q)
        h1 = np.maximum(x @ w["W1"].T + w["b1"], 0)
        h2 = np.maximum(h1 @ w["W2"].T + w["b2"], 0)
        h3 = np.maximum(h2 @ w["W3"].T + w["b3"], 0)
        return np.mean((h3 @ w["W4"] + w["b4"][0] - y) ** 2)

    assert np.isclose(f(pb), loss)
    idx = rng.choice(mlp_ref.NPARAM, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(pb)
        e[i] = h
        fd = (f(pb + e) - f(pb - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), i


def test_neighbour_histogram_brute_force():
    rng = np.random.default_rng(2)
    om = rng.uniform(-0.2, 0.2, (400, 2))
    K = (128, 128)
    moff = [0, 150, 150, 400]
    f, hist = mlp_ref.features(om, K, moff)
    t = om * (128 / (2 * np.pi))
    for s in range(3):
        a, b = moff[s], moff[s + 1]
        for m in range(a, b):
            d = t[a:b] - t[m]
            d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]
            d2[m - a] = np.inf
            d2 = d2[d2 < 4]
            expect = np.bincount(np.minimum((np.sqrt(d2) * 8).astype(int), 15), minlength=16)
            assert np.array_equal(hist[m], expect)
    assert np.allclose(f[:, 2:], np.log1p(hist))
