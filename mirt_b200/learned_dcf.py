"""Learned density compensation: a small MLP that predicts Pipe & Menon weights
from local trajectory geometry (no counterpart in the reference; its targets
come from ``dcf_pipe``, the device restatement of mri/ir_mri_density_comp.m's
'pipe' method).

* ``dcf_features``: per-sample inputs (|omega| / pi, angle / pi, log1p of the
  16-bin neighbour-count histogram within 2 grid cells), on the device;
* ``DcfMLP``: the 18-64-64-64-1 network, BF16 weights / FP32 accumulation,
  trained and evaluated by the library's own kernels;
* ``make_dataset`` / ``train_learned_dcf``: trajectories (golden-angle radial,
  variable-density spirals, random variable-density sets), Pipe-Menon targets
  (30 FP32 P P' w updates with an FP64 ratio update) on batched device plans,
  sub-sampled training rows, held-out evaluation;
* ``LearnedDCF.predict``: weights for a new trajectory, scaled like the
  reference's Pipe-Menon result (sum of the point spread function = prod(N)).

Run ``python -m mirt_b200.learned_dcf --ntraj 10000 --out model.npz`` to build
the full training set and train.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import workloads as wl
from ._lib import check, load
from .dcf import dcf_pipe
from .nufft import NufftPlan, _stream_ptr, _torch

NFEAT = 18
HID = 64
NPARAM = HID * NFEAT + HID + 2 * (HID * HID + HID) + HID + 1
_fp = C.POINTER(C.c_float)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


def he_init(seed: int = 0) -> np.ndarray:
    """He-uniform weights (limit sqrt(6 / fan_in)), zero biases, FP32."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((NFEAT, HID), (HID, HID), (HID, HID), (HID, 1)):
        lim = np.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, fan_out * fan_in))
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts).astype(np.float32)


def dcf_features(om_dev, K, slice_moff=None, stream=None):
    """Device FP32 [M, 18] features of the 2D samples om_dev (device FP64 [M, 2])."""
    torch = _torch()
    lib = load()
    om_dev = om_dev.to(dtype=torch.float64)
    M = om_dev.shape[0]
    omc = om_dev.t().contiguous()                       # [2, M] = column-major [M, 2]
    feat = torch.empty((M, NFEAT), dtype=torch.float32, device=om_dev.device)
    Ka = np.ascontiguousarray(np.asarray(K, dtype=np.int32))
    if slice_moff is None:
        mo, ns = None, 1
    else:
        mo = np.ascontiguousarray(np.asarray(slice_moff, dtype=np.int64))
        ns = len(mo) - 1
    check(lib.mirt_dcf_features(C.c_void_p(omc.data_ptr()), M,
                                None if mo is None else mo.ctypes.data_as(_i64p), ns,
                                Ka.ctypes.data_as(_i32p), C.c_void_p(feat.data_ptr()),
                                _stream_ptr(stream)))
    return feat


class DcfMLP:
    """The regressor behind ``mirt_mlp_*``: parameters live on the device."""

    def __init__(self, params=None, seed=0):
        self.lib = load()
        p = he_init(seed) if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p.size != NPARAM:
            raise ValueError(f"expected {NPARAM} parameters")
        h = C.c_void_p()
        check(self.lib.mirt_mlp_create(C.byref(h), p.ctypes.data_as(_fp)))
        self.handle = h

    def params(self) -> np.ndarray:
        out = np.empty(NPARAM, dtype=np.float32)
        check(self.lib.mirt_mlp_params(self.handle, out.ctypes.data_as(_fp)))
        return out

    def grad(self, x, y, stream=None):
        """(loss, gradient) of the mean squared error over all rows."""
        g = np.empty(NPARAM, dtype=np.float32)
        loss = C.c_float()
        check(self.lib.mirt_mlp_grad(self.handle, C.c_void_p(x.data_ptr()),
                                     C.c_void_p(y.data_ptr()), x.shape[0], g.ctypes.data_as(_fp),
                                     C.byref(loss), _stream_ptr(stream)))
        return float(loss.value), g

    def train(self, x, y, steps, batch=8192, lr=1e-3, seed=0, stream=None):
        """Adam steps on rows drawn from (x, y); returns the loss per step."""
        hist = np.zeros(max(steps, 1), dtype=np.float32)
        check(self.lib.mirt_mlp_train(self.handle, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(y.data_ptr()), x.shape[0], int(batch), int(steps),
                                      float(lr), int(seed), hist.ctypes.data_as(_fp),
                                      _stream_ptr(stream)))
        return hist[:steps]

    def infer(self, x, mu=0.0, sigma=1.0, weights=True, stream=None):
        """Network output (weights=False) or w = exp(sigma * out + mu) (FP64)."""
        torch = _torch()
        n = x.shape[0]
        if weights:
            w = torch.empty(n, dtype=torch.float64, device=x.device)
            check(self.lib.mirt_mlp_infer(self.handle, C.c_void_p(x.data_ptr()), n, float(mu),
                                          float(sigma), None, C.c_void_p(w.data_ptr()),
                                          _stream_ptr(stream)))
        else:
            w = torch.empty(n, dtype=torch.float32, device=x.device)
            check(self.lib.mirt_mlp_infer(self.handle, C.c_void_p(x.data_ptr()), n, float(mu),
                                          float(sigma), C.c_void_p(w.data_ptr()), None,
                                          _stream_ptr(stream)))
        return w

    def set_tensor_cores(self, on=True):
        """Inference on the tensor cores (the default) or on the FP32 pipes."""
        check(self.lib.mirt_mlp_set_tensor_cores(self.handle, int(bool(on))))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mirt_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# trajectories, targets, training
# ---------------------------------------------------------------------------
def trajectory(i: int, seed: int, N: int, nro: int = None, spiral_samples: int = None,
               radial=(32, 512), spiral=(8, 48), random_m=(20000, 200000)):
    """Trajectory i of the seeded family mix: i mod 3 = 0 golden-angle radial
    (spokes ~ U{radial}, nro = 2N readout), 1 variable-density spiral
    (interleaves ~ U{spiral}, alpha ~ U[1, 2]), 2 random variable-density set
    (M ~ U{random_m}, gamma ~ U[1.2, 2])."""
    rng = np.random.default_rng([seed, i])
    nro = 2 * N if nro is None else nro
    fam = i % 3
    if fam == 0:
        ns = int(rng.integers(radial[0], radial[1] + 1))
        return wl.ga_radial(ns, nro, start=rng.uniform(0, np.pi))
    if fam == 1:
        nint = int(rng.integers(spiral[0], spiral[1] + 1))
        ns = 16 * N if spiral_samples is None else spiral_samples
        return wl.vd_spiral(nint, ns, N, alpha=rng.uniform(1.0, 2.0))
    M = int(rng.integers(random_m[0], random_m[1] + 1))
    return wl.vd_random(M, rng, gamma=rng.uniform(1.2, 2.0))


def pipe_targets(oms, N, K, niter=29, J=6, L=1024, stream=None):
    """Pipe-Menon weights (niter + 1 = 30 updates, thresh 0) of the
    trajectories in one batched single-column plan; returns (w device FP64,
    slice offsets, om device FP64 [M, 2])."""
    torch = _torch()
    moff = np.concatenate([[0], np.cumsum([len(o) for o in oms])]).astype(np.int64)
    om = np.concatenate(oms)
    G = NufftPlan(om, (N, N), (J, J), (K, K), n_shift=(N / 2, N / 2), Ld=L, ncol=1,
                  slice_moff=moff, stream=stream)
    w = dcf_pipe(G, niter=niter, thresh=0.0, stream=stream)
    return w, moff, torch.from_numpy(om).cuda(), G


def make_dataset(ntraj, seed=0, N=256, K=512, rows_per_traj=2048, batch_samples=24_000_000,
                 niter=29, holdout=0.1, traj_kw=None, verbose=False):
    """Features / log-weight rows of the training trajectories (sub-sampled
    per trajectory) and the held-out trajectories kept whole."""
    torch = _torch()
    traj_kw = traj_kw or {}
    n_hold = max(1, int(round(ntraj * holdout)))
    n_train = ntraj - n_hold
    xs, ys, held = [], [], []
    i = 0
    t0 = time.perf_counter()
    while i < ntraj:
        # one batched plan: trajectories until the next would pass batch_samples
        oms, tot = [], 0
        while i < ntraj:
            o = trajectory(i, seed, N, **traj_kw)
            if oms and tot + len(o) > batch_samples:
                break
            oms.append(o)
            tot += len(o)
            i += 1
        first = i - len(oms)
        w, moff, omd, G = pipe_targets(oms, N, K, niter=niter)
        feat = dcf_features(omd, (K, K), moff)
        logw = torch.log(w).to(torch.float32)
        g = torch.Generator(device="cpu").manual_seed(seed * 7919 + first)
        for j in range(len(oms)):
            a, b = int(moff[j]), int(moff[j + 1])
            if first + j < n_train:
                k = min(rows_per_traj, b - a)
                sel = torch.randperm(b - a, generator=g)[:k].cuda() + a
                xs.append(feat[sel])
                ys.append(logw[sel])
            else:
                held.append(dict(om=oms[j], w=w[a:b].clone(), feat=feat[a:b].clone()))
        del G
        if verbose:
            print(f"  trajectories {i}/{ntraj}, {time.perf_counter() - t0:.1f} s", flush=True)
    x = torch.cat(xs) if xs else torch.empty((0, NFEAT), device="cuda")
    y = torch.cat(ys) if ys else torch.empty(0, device="cuda")
    return x.contiguous(), y.contiguous(), held


class LearnedDCF:
    """Trained regressor plus the standardisation of its log-weight targets."""

    def __init__(self, mlp: DcfMLP, mu: float, sigma: float, N: int, K: int):
        self.mlp, self.mu, self.sigma, self.N, self.K = mlp, mu, sigma, N, K

    def predict(self, om, G: NufftPlan | None = None, slice_moff=None):
        """Device FP64 weights for om (numpy [M, 2] radians or device tensor);
        with G (single-column plan of the same samples) they are scaled so that
        sum(real(G' w)) = prod(N) per slice, like Pipe-Menon's result."""
        torch = _torch()
        omd = om if hasattr(om, "data_ptr") else torch.from_numpy(np.asarray(om, np.float64)).cuda()
        feat = dcf_features(omd, (self.K, self.K), slice_moff)
        w = self.mlp.infer(feat, self.mu, self.sigma)
        if G is not None:
            w = scale_psf(G, w)
        return w

    def save(self, path):
        np.savez(path, params=self.mlp.params(), mu=self.mu, sigma=self.sigma, N=self.N, K=self.K)

    @staticmethod
    def pretrained(N: int = 256, K: int = 512):
        """The regressor trained by ``python -m mirt_b200.learned_dcf --ntraj 10000
        --steps 20000 --batch 16384`` (seed 0), shipped in mirt_b200/data."""
        import os
        path = os.path.join(os.path.dirname(__file__), "data", f"learned_dcf_n{N}_k{K}.npz")
        return LearnedDCF.load(path)

    @staticmethod
    def load(path):
        z = np.load(path)
        return LearnedDCF(DcfMLP(z["params"]), float(z["mu"]), float(z["sigma"]), int(z["N"]),
                          int(z["K"]))


def scale_psf(G: NufftPlan, w, fov=1.0, stream=None):
    """w * prod(N ./ fov) / sum(real(G' w)) per slice (the reference's
    Pipe-Menon scaling, mri/ir_mri_density_comp.m:258-261), in place."""
    fv = np.ascontiguousarray(np.broadcast_to(np.asarray(fov, dtype=np.float64), (G.D,)))
    check(G.lib.mirt_dcf_scale(G.handle, C.c_void_p(w.data_ptr()),
                               fv.ctypes.data_as(C.POINTER(C.c_double)), _stream_ptr(stream)))
    return w


def train_learned_dcf(x, y, steps=4000, batch=8192, lr=2e-3, seed=0, N=256, K=512):
    """Standardise the log-weight targets and train; returns (LearnedDCF, losses)."""
    mu = float(y.mean())
    sigma = float(y.std())
    yn = ((y - mu) / sigma).contiguous()
    mlp = DcfMLP(seed=seed)
    losses = mlp.train(x, yn, steps, batch=batch, lr=lr, seed=seed)
    return LearnedDCF(mlp, mu, sigma, N, K), losses


def nrmse(a, b):
    a = a.to(dtype=b.dtype)
    return float((a - b).norm() / b.norm())


def evaluate(model: LearnedDCF, held, N, K, seed=0):
    """Held-out weight NRMSE and adjoint-reconstruction NRMSE against the
    Pipe-Menon weights (recon = G'(w .* G x) of a seeded ellipse phantom)."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    out = []
    for h in held:
        G = NufftPlan(h["om"], (N, N), (6, 6), (K, K), n_shift=(N / 2, N / 2), Ld=1024, ncol=1)
        wp = model.predict(h["om"], G)
        img = wl.ellipses(N, 10, rng).astype(np.complex64)
        x = torch.from_numpy(np.ascontiguousarray(img.T)[None, :, :, None]).cuda()
        yk = G.forward(x)
        r_p = G.adjoint((yk * h["w"].to(torch.complex64)[:, None]).contiguous())
        r_m = G.adjoint((yk * wp.to(torch.complex64)[:, None]).contiguous())
        out.append(dict(M=len(h["om"]), w_nrmse=nrmse(wp, h["w"]), recon_nrmse=nrmse(r_m, r_p)))
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--ntraj", type=int, default=10000)
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--K", type=int, default=512)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--rows", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="learned_dcf.npz")
    a = ap.parse_args()
    t0 = time.perf_counter()
    x, y, held = make_dataset(a.ntraj, a.seed, a.N, a.K, rows_per_traj=a.rows, verbose=True)
    t1 = time.perf_counter()
    model, losses = train_learned_dcf(x, y, a.steps, a.batch, a.lr, a.seed, a.N, a.K)
    t2 = time.perf_counter()
    ev = evaluate(model, held, a.N, a.K, a.seed)
    model.save(a.out)
    summ = dict(ntraj=a.ntraj, rows=int(x.shape[0]), dataset_s=t1 - t0, train_s=t2 - t1,
                loss_first=float(losses[0]), loss_last=float(np.mean(losses[-50:])),
                heldout=len(ev), w_nrmse=float(np.median([e["w_nrmse"] for e in ev])),
                recon_nrmse=float(np.median([e["recon_nrmse"] for e in ev])))
    print(json.dumps(summ))


if __name__ == "__main__":
    main()
