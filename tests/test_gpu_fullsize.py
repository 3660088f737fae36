"""GPU parity at the benchmark's full sizes, through the plans the benchmark times.

* 2D batch (64 uneven golden-angle slices, 8.39 M samples, 32 coils,
  K = 512^2, J = 6, L = 1024, autotuned): the table gather and the table
  spread of the whole batch in one call each, compared with the reference's
  FP64 kernels (nufft/table/interp2_table1_for.c:24-99,
  interp2_table1_adj.c:24-95) on slice 0, the lightest and the heaviest slice,
  coils 0 and 31; and the full NUFFT forward / adjoint of the batch against
  the FP64 glue (nufft/nufft.m:128-165, nufft/nufft_adj.m:32-80) on the same
  slices and coils.
* 3D kooshball (16,384 spokes x 256, 4.19 M samples, 8 coils, K = 256^3,
  J = 6, L = 512, autotuned): the gather on a seeded 4,096-sample subset of
  the full call's output (coils 0 and 7), and the full adjoint of every sample
  for coils 0 and 7 (interp3_table1_for.c:24-130, interp3_table1_adj.c:24-121),
  which crosses the dense k-space centre.
* Per configuration, the NUFFT's error against the exact DTFT
  (nufft/dtft.m:80-112, nufft/dtft_adj.m:40-60) stays within 1.5x the FP64
  oracle's own error against it (the table's quantisation) plus 1e-6.

Tolerances as everywhere: relative L2 <= 1e-6 forward, <= 1e-5 adjoint.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import mirt_b200 as mb
import oracle
from oracle import nufft_ref as nr
from conftest import ref_impl, rel_l2
import fullsize as fs

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-6
ADJ_TOL = 1e-5


def _interp_calls(plan, torch):
    """gather(grid) -> samples and spread(samples) -> grid through the
    plan's interpolation plan (the C ABI's mirt_interp_plan_forward/adjoint)."""
    from mirt_b200._lib import check
    ip = plan.lib.mirt_nufft_interp_plan(plan.handle)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def gather(grid, out):
        check(plan.lib.mirt_interp_plan_forward(ip, C.c_void_p(grid.data_ptr()),
                                                C.c_void_p(out.data_ptr()), st))

    def spread(fm, out):
        check(plan.lib.mirt_interp_plan_adjoint(ip, C.c_void_p(fm.data_ptr()),
                                                C.c_void_p(out.data_ptr()), st))
    return gather, spread


def _randn(torch, shape, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.randn(shape, dtype=torch.complex64, device="cuda", generator=g)


@pytest.fixture(scope="module")
def c2_plan():
    om, moff, spokes = fs.c2_trajectory()
    w = fs.C2
    N, K = w["N"], w["K"]
    plan = mb.NufftPlan(om, (N, N), (6, 6), (K, K), n_shift=(N / 2, N / 2), Ld=w["L"],
                        ncol=w["ncoil"], slice_moff=moff)
    cfg = plan.autotune()
    yield plan, cfg, om, moff, spokes
    plan.close()


def _c2_slices(spokes):
    return sorted({0, int(np.argmin(spokes)), int(np.argmax(spokes))})


def test_c2_interp_full_batch_vs_reference(c2_plan):
    import torch
    plan, cfg, om, moff, spokes = c2_plan
    # the benchmarked path: TMA-staged gather and row-sweep spread
    assert cfg["gather_tma"] in (1, 2) and cfg["spread_sweep"] != 0, cfg
    w = fs.C2
    K = w["K"]
    gather, spread = _interp_calls(plan, torch)
    grid = _randn(torch, (plan.nslice, K, K, w["ncoil"]), 21)
    X = torch.empty(plan.sample_shape, dtype=torch.complex64, device="cuda")
    gather(grid, X)
    fm = _randn(torch, plan.sample_shape, 22)
    out = torch.empty_like(grid)
    spread(fm, out)
    torch.cuda.synchronize()
    h = [mb.minmax_kb_table(w["N"], 6, K, w["L"])] * 2
    ns = np.array([w["N"] / 2] * 2)
    for s in _c2_slices(spokes):
        sl = slice(int(moff[s]), int(moff[s + 1]))
        oms = om[sl]
        tm = oms / (2 * np.pi / K)
        ph = np.exp(1j * (oms @ ns))
        Xs = X[sl].cpu().numpy()
        fms = fm[sl].cpu().numpy()
        for c in (0, w["ncoil"] - 1):
            ck = grid[s, :, :, c].cpu().numpy().reshape(-1)       # k1 + K1 k2
            ref = oracle.interp_for(ck, h, [6, 6], [w["L"]] * 2, tm, [K, K], 0,
                                    impl=ref_impl())[:, 0] * ph
            assert rel_l2(Xs[:, c], ref) <= FWD_TOL, (s, c)
            ref_a = oracle.interp_adj(fms[:, c] * np.conj(ph), h, [6, 6], [w["L"]] * 2, tm,
                                      [K, K], 0, impl=ref_impl())[:, 0]
            got = out[s, :, :, c].cpu().numpy().reshape(-1)
            assert rel_l2(got, ref_a) <= ADJ_TOL, (s, c)


def test_c2_nufft_full_batch_vs_oracle(c2_plan):
    import torch
    plan, cfg, om, moff, spokes = c2_plan
    w = fs.C2
    N, K = w["N"], w["K"]
    x = _randn(torch, plan.image_shape, 23)
    X = plan.forward(x)
    y = _randn(torch, plan.sample_shape, 24)
    xa = plan.adjoint(y)
    torch.cuda.synchronize()
    imp = ref_impl()
    fw = lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                         impl=imp)[:, 0]
    ad = lambda Y, s: oracle.interp_adj(Y, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                        impl=imp)[:, 0]
    for s in _c2_slices(spokes):
        sl = slice(int(moff[s]), int(moff[s + 1]))
        st_o = nr.nufft_init_table(om[sl], (N, N), (6, 6), (K, K), (N / 2, N / 2), w["L"])
        for c in (0, w["ncoil"] - 1):
            img = x[s, :, :, c].cpu().numpy().T                   # [n1, n2]
            assert rel_l2(X[sl, c].cpu().numpy(), nr.nufft(img, st_o, fw)) <= FWD_TOL, (s, c)
            ref = nr.nufft_adj(y[sl, c].cpu().numpy(), st_o, ad)
            assert rel_l2(xa[s, :, :, c].cpu().numpy().T, ref) <= ADJ_TOL, (s, c)


@pytest.fixture(scope="module")
def c3_plan():
    om = fs.c3_trajectory()
    w = fs.C3
    N, K = w["N"], w["K"]
    plan = mb.NufftPlan(om, (N,) * 3, (6,) * 3, (K,) * 3, n_shift=(N / 2,) * 3, Ld=w["L"],
                        ncol=w["ncoil"])
    cfg = plan.autotune()
    yield plan, cfg, om
    plan.close()


def test_c3_interp_full_vs_reference(c3_plan):
    import torch
    plan, cfg, om = c3_plan
    w = fs.C3
    K, L = w["K"], w["L"]
    gather, spread = _interp_calls(plan, torch)
    grid = _randn(torch, (1, K, K, K, w["ncoil"]), 31)
    X = torch.empty(plan.sample_shape, dtype=torch.complex64, device="cuda")
    gather(grid, X)
    fm = _randn(torch, plan.sample_shape, 32)
    out = torch.empty_like(grid)
    spread(fm, out)
    torch.cuda.synchronize()
    h = [mb.minmax_kb_table(w["N"], 6, K, L)] * 3
    ns = np.array([w["N"] / 2] * 3)
    tm = om / (2 * np.pi / K)
    ph = np.exp(1j * (om @ ns))
    sub = np.sort(np.random.default_rng(33).choice(len(om), fs.NSUB, replace=False))
    Xs = X[torch.from_numpy(sub).cuda()].cpu().numpy()
    fmh = fm.cpu().numpy()
    cols = (0, w["ncoil"] - 1)
    for c in cols:
        ck = grid[0, ..., c].cpu().numpy().reshape(-1)            # k1 + K1 (k2 + K2 k3)
        ref = oracle.interp_for(ck, h, [6] * 3, [L] * 3, tm[sub], [K] * 3, 0,
                                impl=ref_impl())[:, 0] * ph[sub]
        assert rel_l2(Xs[:, c], ref) <= FWD_TOL, c
    # the full adjoint of every sample, both columns at once (one thread each)
    Y = fmh[:, list(cols)] * np.conj(ph)[:, None]
    ref_a = oracle.interp_adj(Y, h, [6] * 3, [L] * 3, tm, [K] * 3, 0, impl=ref_impl(),
                              nthreads=2)
    for i, c in enumerate(cols):
        got = out[0, ..., c].cpu().numpy().reshape(-1)
        assert rel_l2(got, ref_a[:, i]) <= ADJ_TOL, c


def test_c3_nufft_vs_oracle(c3_plan):
    """Full 3D NUFFT of the whole kooshball, coil 0: forward on the
    4,096-sample subset, adjoint of every sample."""
    import torch
    plan, cfg, om = c3_plan
    w = fs.C3
    N, K, L = w["N"], w["K"], w["L"]
    x = _randn(torch, plan.image_shape, 34)
    X = plan.forward(x)
    y = _randn(torch, plan.sample_shape, 35)
    xa = plan.adjoint(y)
    torch.cuda.synchronize()
    imp = ref_impl()
    sub = np.sort(np.random.default_rng(36).choice(len(om), fs.NSUB, replace=False))
    img = np.transpose(x[0, ..., 0].cpu().numpy(), (2, 1, 0))     # [n1, n2, n3]
    st_s = nr.nufft_init_table(om[sub], (N,) * 3, (6,) * 3, (K,) * 3, (N / 2,) * 3, L)
    fw = lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                         impl=imp)[:, 0]
    Xsub = X[torch.from_numpy(sub).cuda(), 0].cpu().numpy()
    assert rel_l2(Xsub, nr.nufft(img, st_s, fw)) <= FWD_TOL
    st_o = nr.nufft_init_table(om, (N,) * 3, (6,) * 3, (K,) * 3, (N / 2,) * 3, L)
    ad = lambda Y, s: oracle.interp_adj(Y, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                        impl=imp)[:, 0]
    ref = nr.nufft_adj(y[:, 0].cpu().numpy(), st_o, ad)
    got = np.transpose(xa[0, ..., 0].cpu().numpy(), (2, 1, 0))
    assert rel_l2(got, ref) <= ADJ_TOL


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_dtft_error_per_config(name):
    r = fs.dtft_accuracy(name)
    print(r)
    assert r["fwd_gpu_oracle"] <= FWD_TOL and r["adj_gpu_oracle"] <= ADJ_TOL, r
    assert r["fwd_gpu_dtft"] <= 1.5 * r["fwd_oracle_dtft"] + 1e-6, r
    assert r["adj_gpu_dtft"] <= 1.5 * r["adj_oracle_dtft"] + 1e-6, r
