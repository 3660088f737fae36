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


@pytest.mark.parametrize("C,K1", [(32, 80), (40, 82)])
def test_32coil_row_sweep_adjoint_vs_oracle(C, K1):
    """32-coil chunks: the plan's default spread is the row sweep.  The NUFFT
    adjoint against the oracle for several band / segment choices (K1 = 80
    and 82, segment edges anywhere), bitwise the same for all of them, and
    against the tiled spread to FP32 rounding; a newfft plan of the same
    batch (grid phase on the transpose) against its oracle."""
    import torch
    from oracle import newfft_ref as nf
    rng = np.random.default_rng(40 + C)
    N, K = (40, 48), (K1, 96)
    counts = [1200, 2500, 700]
    moff = np.concatenate([[0], np.cumsum(counts)])
    om = np.concatenate([rng.uniform(-np.pi, np.pi, (c, 2)) for c in counts])
    ns = (20, 24)
    plan = mb.NufftPlan(om, N, (6, 6), K, n_shift=ns, Ld=1024, ncol=C, slice_moff=moff)
    assert plan.config()["spread_sweep"] == -1     # balanced teams by default
    plan.set_dense(False)                        # (bands of 1, 2, 4 rows below: the same sums)
    X = rng.standard_normal((len(om), C)) + 1j * rng.standard_normal((len(om), C))
    Xd = torch.from_numpy(X.astype(np.complex64)).cuda()
    out = plan.adjoint(Xd).cpu().numpy()
    refs = []
    for s in range(len(counts)):
        sl = slice(moff[s], moff[s + 1])
        st_o = nr.nufft_init_table(om[sl], N, (6, 6), K, ns, 1024)
        _, ad = _oracle_pair(st_o)
        refs.append({c: nr.nufft_adj(X[sl, c], st_o, ad) for c in (0, 17, C - 1)})
    for seg, rows in [(None, None), (3, 2), (5, 1), (1, 4), (-1, 2)]:
        if seg is not None:
            plan.set_sweep(seg, rows)
        o = plan.adjoint(Xd).cpu().numpy()
        for s in range(len(counts)):
            for c, ref in refs[s].items():
                assert rel_l2(o[s, :, :, c].T, ref) <= ADJ_TOL, (seg, rows, s, c)
        assert np.array_equal(o, out)          # same sums for every band / segment choice
    assert np.array_equal(out, plan.adjoint(Xd).cpu().numpy())
    plan.set_sweep(0)
    assert rel_l2(plan.adjoint(Xd).cpu().numpy(), out) <= 5e-6
    plan.close()
    nplan = mb.newfft(om, N, Kd=K, n_shift=ns, ncol=C, slice_moff=moff)
    outn = nplan.adjoint(Xd).cpu().numpy()
    for s in range(len(counts)):
        sl = slice(moff[s], moff[s + 1])
        so = nf.newfft_init(om[sl], N, Kd=K, n_shift=ns)
        assert rel_l2(outn[s, :, :, C - 1].T, nf.newfft_adj(X[sl, C - 1], so)) <= ADJ_TOL, s
    nplan.close()


@pytest.mark.parametrize("C,nslice", [(32, 5), (32, 11), (8, 11)])
def test_host_calls_pipelined_by_slice_chunks(C, nslice):
    """Host-buffer calls of a multi-slice plan run in slice chunks (copies on
    their own streams overlapping the compute; 11 slices: five chunks of two
    and one of one).  Their results are the device calls' to FP32 rounding
    (the chunk FFT plans have other batch counts); the adjoint is chunked
    where the spread is the row sweep (32 coils), whole-batch otherwise."""
    import torch
    rng = np.random.default_rng(60 + nslice + C)
    N, K = (32, 40), (64, 80)
    counts = rng.integers(300, 1200, nslice)
    moff = np.concatenate([[0], np.cumsum(counts)])
    om = rng.uniform(-np.pi, np.pi, (int(moff[-1]), 2))
    for s in (0, nslice - 1):                   # dense bins (patches) in the first and last chunk
        om[moff[s]:moff[s] + 200] = rng.uniform(-0.05, 0.05, (200, 2))
    plan = mb.NufftPlan(om, N, (6, 6), K, n_shift=(16, 20), Ld=1024, ncol=C, slice_moff=moff)
    x = (rng.standard_normal(plan.image_shape) + 1j * rng.standard_normal(plan.image_shape))
    x = x.astype(np.complex64)
    for _ in range(2):                          # the second call reuses streams and plans
        a = plan.forward_host(x)
        b = plan.forward(torch.from_numpy(x).cuda()).cpu().numpy()
        assert rel_l2(a, b) <= 1e-6
        y = plan.adjoint_host(b)
        z = plan.adjoint(torch.from_numpy(b).cuda()).cpu().numpy()
        assert rel_l2(y, z) <= 1e-6
    for s in (0, nslice - 1):                   # first and last chunk against the oracle
        sl = slice(moff[s], moff[s + 1])
        st_o = nr.nufft_init_table(om[sl], N, (6, 6), K, (16, 20), 1024)
        fw, ad = _oracle_pair(st_o)
        assert rel_l2(a[sl, C - 1], nr.nufft(x[s, :, :, C - 1].T, st_o, fw)) <= FWD_TOL
        assert rel_l2(y[s, :, :, 0].T, nr.nufft_adj(b[sl, 0], st_o, ad)) <= ADJ_TOL
    plan.close()


@pytest.mark.parametrize("ktype,params", [("kaiser", ()), ("kaiser", ([15.0, 15.0], [1, 1])),
                                          ("minmax:tuned", ()), ("uniform", ()), ("linear", ())])
def test_nufft_init_other_interpolators(ktype, params):
    """nufft_init(om, Nd, Jd, Kd, n_shift, 'table', L, ktype, ...) for the
    interpolators other than 'minmax:kb': the library's tables and scaling
    factors on the newfft plan with phasing 'complex' against the oracle's
    nufft / nufft_adj with its own restatement of them."""
    rng = np.random.default_rng(17)
    Nd, Jd, Kd = (32, 24), (6, 5), (64, 48)
    om = rng.uniform(-np.pi, np.pi, (600, 2))
    ns = np.array([16.0, 12.0])
    st = mb.nufft_init(om, Nd, Jd, Kd, ns, "table", 2 ** 10, ktype, *params)
    so = nr.nufft_init_table_ktype(om, Nd, Jd, Kd, ns, 2 ** 10, ktype, *params)
    fw, ad = _oracle_pair(so)
    x = rng.standard_normal(Nd) + 1j * rng.standard_normal(Nd)
    X_o = nr.nufft(x, so, fw)
    # the newfft plan's tolerance (1e-5 each way, its FP32 FFT included)
    assert rel_l2(mb.nufft(x, st), X_o) <= 1e-5
    assert rel_l2(mb.nufft_adj(X_o, st), nr.nufft_adj(X_o, so, ad)) <= 1e-5


def test_nufft_init_kaiser_3d_table_test_setup():
    """nufft/nufft_table_test.m's 3D 'kaiser' set-up (Jd = [3 4 3], odd and
    even J, n_shift = [3 7 2], Ld = [2^8 2^7 2^7]) on the device against the
    oracle, forward and adjoint."""
    Jd, Nd = (3, 4, 3), (10, 8, 9)
    Kd = tuple(2 * np.asarray(Nd))
    ns = np.array([3.0, 7.0, 2.0])
    gam = 2 * np.pi / np.asarray(Kd)
    g = np.meshgrid(*[np.linspace(-2 * k, 2 * k, n) for k, n in zip(Kd, (21, 18, 23))],
                    indexing="ij")
    om = np.stack([gam[d] * g[d].ravel(order="F") for d in range(3)], 1)
    Ld = (2 ** 8, 2 ** 7, 2 ** 7)
    st = mb.nufft_init(om, Nd, Jd, Kd, ns, "table", Ld, "kaiser")
    so = nr.nufft_init_table_ktype(om, Nd, Jd, Kd, ns, Ld, "kaiser")
    fw, ad = _oracle_pair(so)
    rng = np.random.default_rng(8)
    x = rng.standard_normal(Nd) + 1j * rng.standard_normal(Nd)
    X_o = nr.nufft(x, so, fw)
    assert rel_l2(mb.nufft(x, st), X_o) <= 1e-5
    X = np.arange(1, len(om) + 1) + 1j
    assert rel_l2(mb.nufft_adj(X, st), nr.nufft_adj(X, so, ad)) <= 1e-5
