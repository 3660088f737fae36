"""FP64 restatement of the learned density compensation's features and network.

TEST INFRASTRUCTURE ONLY (the checker of mirt_dcf_features and mirt_mlp_*).

* ``features``: the per-sample inputs (radius, angle, log1p of the 16-bin
  neighbour-count histogram within 2 grid cells), with the same FP64 distance
  formula and exact bin edges as the device kernel;
* ``forward`` / ``grad``: the 18-64-64-64-1 ReLU network on the BF16
  rounding of the parameters, in FP64, and the gradient of the mean squared
  error by explicit back-propagation.
"""
from __future__ import annotations

import numpy as np

NFEAT = 18
HID = 64
NPARAM = HID * NFEAT + HID + 2 * (HID * HID + HID) + HID + 1
_EDGES2 = np.array([(e * 0.125) ** 2 for e in range(1, 16)])


def bf16_round(x) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p)
    o = 0
    out = {}
    for name, shape in (("W1", (HID, NFEAT)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
                        ("W3", (HID, HID)), ("b3", (HID,)), ("W4", (HID,)), ("b4", (1,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def init_params(rng: np.random.Generator) -> np.ndarray:
    """He-uniform weights, zero biases, FP32."""
    parts = []
    for fan_in, fan_out in ((NFEAT, HID), (HID, HID), (HID, HID), (HID, 1)):
        lim = np.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, fan_out * fan_in))
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts).astype(np.float32)


def forward(p, x):
    """Network output for rows x [n, 18] with BF16-rounded parameters (FP64 math)."""
    w = {k: v.astype(np.float64) for k, v in unpack(bf16_round(p)).items()}
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ w["W1"].T + w["b1"], 0)
    h2 = np.maximum(h1 @ w["W2"].T + w["b2"], 0)
    h3 = np.maximum(h2 @ w["W3"].T + w["b3"], 0)
    return h3 @ w["W4"] + w["b4"][0], (h1, h2, h3)


def grad(p, x, y):
    """(loss, gradient [NPARAM]) of mean((out - y)^2) w.r.t. the parameters,
    evaluated at their BF16 rounding."""
    w = {k: v.astype(np.float64) for k, v in unpack(bf16_round(p)).items()}
    x = np.asarray(x, dtype=np.float64)
    out, (h1, h2, h3) = forward(p, x)
    n = x.shape[0]
    r = out - np.asarray(y, dtype=np.float64)
    loss = np.mean(r * r)
    dout = 2 * r / n
    d3 = (h3 > 0) * np.outer(dout, w["W4"])
    d2 = (h2 > 0) * (d3 @ w["W3"])
    d1 = (h1 > 0) * (d2 @ w["W2"])
    g = [d1.T @ x, d1.sum(0), d2.T @ h1, d2.sum(0), d3.T @ h2, d3.sum(0), h3.T @ dout,
         np.array([dout.sum()])]
    return loss, np.concatenate([a.ravel() for a in g])


def features(om, K, slice_moff=None):
    """[M, 18] FP64 features of 2D samples om [M, 2] (radians)."""
    from scipy.spatial import cKDTree
    om = np.asarray(om, dtype=np.float64)
    M = om.shape[0]
    moff = [0, M] if slice_moff is None else list(slice_moff)
    t = np.stack([om[:, 0] * (K[0] / (2 * np.pi)), om[:, 1] * (K[1] / (2 * np.pi))], 1)
    hist = np.zeros((M, 16))
    for s in range(len(moff) - 1):
        a, b = moff[s], moff[s + 1]
        if b - a < 2:
            continue
        ts = t[a:b]
        pairs = cKDTree(ts).query_pairs(2.0 + 1e-9, output_type="ndarray")
        if len(pairs) == 0:
            continue
        dx = ts[pairs[:, 1], 0] - ts[pairs[:, 0], 0]
        dy = ts[pairs[:, 1], 1] - ts[pairs[:, 0], 1]
        d2 = dx * dx + dy * dy
        keep = d2 < 4.0
        pairs, d2 = pairs[keep], d2[keep]
        bins = (d2[:, None] >= _EDGES2[None, :]).sum(1)
        np.add.at(hist, (a + pairs[:, 0], bins), 1)
        np.add.at(hist, (a + pairs[:, 1], bins), 1)
    f = np.empty((M, NFEAT))
    f[:, 0] = np.sqrt(om[:, 0] ** 2 + om[:, 1] ** 2) / np.pi
    f[:, 1] = np.arctan2(om[:, 1], om[:, 0]) / np.pi
    f[:, 2:] = np.log1p(hist)
    return f, hist
