"""GPU parity of the full table NUFFT (deapodisation + zero-pad + cuFFT +
gather, and its adjoint) against the FP64 oracle of nufft.m / nufft_adj.m,
plus the error of both against the exact DTFT (reported, and bounded by the
table quantisation)."""
from __future__ import annotations

import numpy as np
import pytest

import mirt_b200 as mb
import oracle
from oracle import nufft_ref as nr
from conftest import ref_impl, rel_l2

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-6
ADJ_TOL = 1e-5


def _radial(nspoke, nread):
    r = np.linspace(-np.pi, np.pi, nread, endpoint=False)
    ang = np.arange(nspoke) * np.pi / nspoke
    return np.stack([np.outer(np.cos(ang), r).ravel(), np.outer(np.sin(ang), r).ravel()], 1)


def _ellipses(N, n, rng):
    """n seeded random ellipses, amplitude U[0,1], phase U[-pi, pi)."""
    y, x = np.meshgrid(np.linspace(-1, 1, N), np.linspace(-1, 1, N), indexing="ij")
    img = np.zeros((N, N), complex)
    for _ in range(n):
        cx, cy = rng.uniform(-0.5, 0.5, 2)
        rx, ry = rng.uniform(0.05, 0.4, 2)
        th = rng.uniform(0, np.pi)
        a = rng.uniform(0, 1) * np.exp(1j * rng.uniform(-np.pi, np.pi))
        xr = (x - cx) * np.cos(th) + (y - cy) * np.sin(th)
        yr = -(x - cx) * np.sin(th) + (y - cy) * np.cos(th)
        img[(xr / rx) ** 2 + (yr / ry) ** 2 <= 1] += a
    return img.T


def _oracle_pair(st):
    imp = ref_impl()
    fw = lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                         impl=imp)[:, 0]
    ad = lambda X, s: oracle.interp_adj(X, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                        impl=imp)[:, 0]
    return fw, ad


def test_c1_config_vs_oracle_and_dtft():
    """64x64 image of 10 ellipses, K=128^2, J=6, L=1024, 64 radial spokes x 128."""
    rng = np.random.default_rng(0)
    N, K = (64, 64), (128, 128)
    om = _radial(64, 128)
    ns = (32, 32)
    x = _ellipses(64, 10, rng)
    st_o = nr.nufft_init_table(om, N, (6, 6), K, ns, 1024)
    fw, ad = _oracle_pair(st_o)
    X_o = nr.nufft(x, st_o, fw)
    st = mb.nufft_init(om, N, (6, 6), K, ns, "table", 1024, "minmax:kb")
    X = mb.nufft(x, st)
    assert rel_l2(X, X_o) <= FWD_TOL
    Xe = nr.dtft(x, om, ns)
    assert rel_l2(X, Xe) < 2e-3 and rel_l2(X_o, Xe) < 2e-3
    y = rng.standard_normal(len(om)) + 1j * rng.standard_normal(len(om))
    xa_o = nr.nufft_adj(y, st_o, ad)
    xa = mb.nufft_adj(y, st)
    assert rel_l2(xa, xa_o) <= ADJ_TOL
    st.close()


def test_multicoil_multislice_vs_oracle():
    import torch
    rng = np.random.default_rng(4)
    N, K = (48, 40), (96, 80)
    C = 8
    counts = [900, 1500, 400]
    moff = np.concatenate([[0], np.cumsum(counts)])
    om = np.concatenate([rng.uniform(-np.pi, np.pi, (c, 2)) for c in counts])
    ns = (24, 20)
    plan = mb.NufftPlan(om, N, (6, 6), K, n_shift=ns, Ld=1024, ncol=C, slice_moff=moff)
    S = len(counts)
    x = rng.standard_normal((S, 40, 48, C)) + 1j * rng.standard_normal((S, 40, 48, C))
    X = rng.standard_normal((len(om), C)) + 1j * rng.standard_normal((len(om), C))
    outF = plan.forward(torch.from_numpy(x.astype(np.complex64)).cuda()).cpu().numpy()
    outA = plan.adjoint(torch.from_numpy(X.astype(np.complex64)).cuda()).cpu().numpy()
    for s in range(S):
        sl = slice(moff[s], moff[s + 1])
        st_o = nr.nufft_init_table(om[sl], N, (6, 6), K, ns, 1024)
        fw, ad = _oracle_pair(st_o)
        for c in range(0, C, 3):
            img = x[s, :, :, c].T
            assert rel_l2(outF[sl, c], nr.nufft(img, st_o, fw)) <= FWD_TOL
            ref = nr.nufft_adj(X[sl, c], st_o, ad)
            assert rel_l2(outA[s, :, :, c].T, ref) <= ADJ_TOL
    plan.close()


def test_host_api_matches_device_api():
    import torch
    rng = np.random.default_rng(8)
    om = _radial(32, 64)
    plan = mb.NufftPlan(om, (32, 32), (6, 6), (64, 64), n_shift=(16, 16), ncol=4)
    x = (rng.standard_normal(plan.image_shape) + 1j * rng.standard_normal(plan.image_shape))
    x = x.astype(np.complex64)
    a = plan.forward_host(x)
    b = plan.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.array_equal(a, b)
    y = plan.adjoint_host(a)
    z = plan.adjoint(torch.from_numpy(a).cuda()).cpu().numpy()
    assert np.array_equal(y, z)
    plan.close()


def test_3d_nufft_vs_oracle():
    rng = np.random.default_rng(12)
    N, K = (16, 12, 10), (32, 24, 20)
    M = 2500
    om = rng.uniform(-np.pi, np.pi, (M, 3))
    ns = tuple(n / 2 for n in N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    st_o = nr.nufft_init_table(om, N, (6, 6, 6), K, ns, 512)
    fw, ad = _oracle_pair(st_o)
    st = mb.nufft_init(om, N, (6, 6, 6), K, ns, "table", 512, "minmax:kb")
    assert rel_l2(mb.nufft(x, st), nr.nufft(x, st_o, fw)) <= FWD_TOL
    y = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    assert rel_l2(mb.nufft_adj(y, st), nr.nufft_adj(y, st_o, ad)) <= ADJ_TOL
    st.close()
