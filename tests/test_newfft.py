"""newfft in table mode on the CPU: the oracle pinned against the exact DTFT
on the reference's own self-test set-up (nufft/newfft.m:589-668: Nd = 21,
20, [20 10], [20 10 8]; om = 3 * 2 pi (rand - 1/2), 100 samples; x0 = rand),
and the library's host table builders against the oracle.

The reference prints max_percent_diff against 'exact' without a threshold;
the bounds here are about 3x the measured errors of the 'kb:minmax' tables
(table0 L = 2^11: <= 0.04 %, table1 L = 2^9: <= 0.003 %).  A wrong phase
convention or sign gives errors of order 100 %.
"""
from __future__ import annotations

import numpy as np
import pytest

import mirt_b200 as mb
from oracle import newfft_ref as nf
from oracle import nufft_ref as nr

ND_LIST = [(21,), (20,), (20, 10), (20, 10, 8)]
BOUND = {"table0": 0.12, "table1": 0.01}       # percent of max |exact|


def _mpd(exact, approx):
    return 100 * np.max(np.abs(approx - exact)) / np.max(np.abs(exact))


def _case(Nd, seed=0):
    rng = np.random.default_rng(seed)
    om = 3 * 2 * np.pi * (rng.random((100, len(Nd))) - 0.5)
    return om, rng.random(Nd)


@pytest.mark.parametrize("Nd", ND_LIST)
@pytest.mark.parametrize("mode", ["table0", "table1"])
def test_oracle_matches_exact_dtft(Nd, mode):
    om, x0 = _case(Nd)
    ns = np.zeros(len(Nd))
    Xe = nr.dtft(x0, om, ns)
    xe = nr.dtft_adj(Xe, om, Nd, ns)
    st = nf.newfft_init(om, Nd, mode=mode)
    assert _mpd(Xe, nf.newfft_for(x0, st)) < BOUND[mode]
    assert _mpd(xe, nf.newfft_adj(Xe, st)) < BOUND[mode]


def test_oracle_n_shift_and_phasing():
    """n_shift = Nd/2 (centred image) with 'real' phasing (Nmid = floor(N/2)),
    and odd N where Nmid differs from (N-1)/2 only for even N."""
    for Nd in [(20, 10), (21, 9)]:
        om, x0 = _case(Nd, 1)
        ns = np.asarray(Nd) / 2
        st = nf.newfft_init(om, Nd, n_shift=ns)
        assert _mpd(nr.dtft(x0, om, ns), nf.newfft_for(x0, st)) < BOUND["table1"]
    assert list(nf.nmid_of((20, 21))) == [10, 10]
    assert list(nf.nmid_of((20, 21), "complex")) == [9.5, 10]


@pytest.mark.parametrize("J,L", [(6, 512), (6, 2048), (5, 7), (8, 64), (2, 1)])
def test_kb_table_builder(J, L):
    h = mb.newfft_kb_table(J, L)
    ref = nf.kb_table(J, L)
    assert h.shape == (J * L + 1,)
    assert np.max(np.abs(h - ref)) <= 1e-13
    assert h[0] == 0 and h[-1] == 0 and np.allclose(h, h[::-1], atol=1e-15)


@pytest.mark.parametrize("N,J,K,nmid", [(20, 6, 40, 10), (21, 6, 42, 10), (64, 6, 128, 32),
                                        (10, 4, 17, 4.5)])
def test_kb_scale_builder(N, J, K, nmid):
    s = mb.newfft_kb_scale(N, J, K, nmid)
    ref = nf.kb_scale(N, J, K, nmid)
    assert np.max(np.abs(s - ref) / np.abs(ref)) <= 1e-12


def test_builder_argument_errors():
    with pytest.raises(mb.MirtError, match="J must be"):
        mb.newfft_kb_table(0, 16)
    with pytest.raises(mb.MirtError, match="positive"):
        mb.newfft_kb_scale(0, 6, 12, 0.0)


def test_newfft_argument_checks_before_any_device_call():
    """Mode, phasing, table and scaling-factor arguments are checked on the
    host first, as newfft.m checks its options."""
    om = np.zeros((4, 2))
    with pytest.raises(ValueError, match="table0"):
        mb.newfft(om, (16, 16), mode="sparse")
    with pytest.raises(ValueError, match="phasing"):
        mb.newfft(om, (16, 16), phasing="flipreal")
    with pytest.raises(ValueError, match="kb_alf and kb_m required"):
        mb.newfft(om, (16, 16), phasing="complex", ktype="kb:user")
    with pytest.raises(ValueError, match="sn is required"):
        mb.newfft(om, (16, 16), tables=[np.ones(6 * 512 + 1)] * 2)


def test_newfft_without_gpu_fails_loudly():
    """No CPU fallback: without a device the plan cannot be made (the device
    stream or the library's device check refuses)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises((mb.MirtError, RuntimeError, AssertionError)):
        mb.newfft(np.zeros((4, 2)), (16, 16))


def test_oracle_complex_tables_without_phases_is_nufft():
    """newfft with the min-max:KB complex tables and sn of nufft_init, no Nmid
    phases and n_shift applied per sample, is the oracle's nufft (the identity
    the GPU test checks for mirt_newfft_create against mirt_nufft_create)."""
    import oracle
    rng = np.random.default_rng(4)
    om = rng.uniform(-np.pi, np.pi, (300, 2))
    Nd, Jd, Kd, ns = (16, 12), (6, 6), (32, 24), np.array([8.0, 6.0])
    st = nr.nufft_init_table(om, Nd, Jd, Kd, ns, 256)
    sn = nr.scaling_factors(Nd, Jd, Kd)
    so = nf.newfft_init(om, Nd, Jd, Kd, n_shift=ns, mode="table0", Ld=256, phasing="complex",
                        h=st["h"], sn=sn)
    so["phase_after"] = np.exp(1j * (om @ ns))          # n_shift only (no Nmid)
    x = rng.standard_normal(Nd) + 1j * rng.standard_normal(Nd)
    fw = lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0)[:, 0]
    a = nf.newfft_for(x, so)
    b = nr.nufft(x, st, fw)
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


@pytest.mark.parametrize("ktype", ["kb:beatty", "diric"])
@pytest.mark.parametrize("Nd", [(21,), (20,), (20, 10), (6,), (6, 5)])
@pytest.mark.parametrize("mode", ["table0", "table1"])
def test_oracle_ktypes_match_exact_dtft(ktype, Nd, mode):
    """The oracle's 'kb:beatty' and 'diric' interpolators (diric with Jd = 2 Nd
    = Kd, as the reference's self-test sets it, nufft/newfft.m:629-635) on the
    self-test set-up, within the same bounds as 'kb:minmax'."""
    Jd = tuple(2 * np.asarray(Nd)) if ktype == "diric" else None
    if Jd is not None and max(Jd) > 16:
        pytest.skip("J > 16")
    om, x0 = _case(Nd)
    ns = np.zeros(len(Nd))
    Xe = nr.dtft(x0, om, ns)
    st = nf.newfft_init(om, Nd, Jd=Jd, mode=mode, ktype=ktype)
    assert _mpd(Xe, nf.newfft_for(x0, st)) < BOUND[mode]
    assert _mpd(nr.dtft_adj(Xe, om, Nd, ns), nf.newfft_adj(Xe, st)) < BOUND[mode]


@pytest.mark.parametrize("ktype", ["kb:minmax", "kb:beatty", "diric"])
@pytest.mark.parametrize("N,J,K,L", [(20, 6, 40, 512), (21, 6, 42, 2048), (6, 12, 12, 512),
                                     (64, 8, 128, 1024)])
def test_ktype_table_and_scale_builders(ktype, N, J, K, L):
    """The library's host builders of the three interpolators against the
    oracle (FP64 both)."""
    nmid = np.floor(N / 2)
    assert np.max(np.abs(mb.newfft_table(ktype, N, J, K, L) - nf.ktype_table(ktype, N, J, K, L))) <= 1e-13
    s, so = mb.newfft_scale(ktype, N, J, K, nmid), nf.ktype_scale(ktype, N, J, K, nmid)
    assert np.max(np.abs(s - so) / np.abs(so)) <= 1e-12


@pytest.mark.parametrize("ktype,N,J,K,L", [
    ("minmax:tuned", 20, 6, 40, 512), ("minmax:tuned", 21, 4, 42, 1024),
    ("minmax:tuned", 16, 8, 32, 256), ("minmax:tuned", 20, 6, 30, 512),
    ("minmax:unif", 20, 6, 40, 512), ("minmax:unif", 21, 5, 32, 256),
    ("linear", 20, 2, 40, 512), ("linear", 21, 4, 42, 256)])
def test_minmax_tuned_unif_linear_builders(ktype, N, J, K, L):
    """'minmax:tuned' (the L = 3 sets for J = 4, 6, L = 2 for J = 8, alpha = 1,
    beta = 0.5 for K/N != 2), 'minmax:unif' and 'linear': the library's builders
    against the oracle (FP64 both; the min-max inverse is Gauss-Jordan in the
    library and LAPACK in numpy)."""
    nmid = np.floor(N / 2)
    h, ho = mb.newfft_table(ktype, N, J, K, L), nf.ktype_table(ktype, N, J, K, L)
    assert np.max(np.abs(h - ho)) <= 1e-11 * np.max(np.abs(ho))
    s, so = mb.newfft_scale(ktype, N, J, K, nmid), nf.ktype_scale(ktype, N, J, K, nmid)
    assert np.max(np.abs(s - so) / np.abs(so)) <= 1e-12


@pytest.mark.parametrize("Nd", [(21,), (20,), (20, 10), (20, 10, 8)])
@pytest.mark.parametrize("mode", ["table0", "table1"])
def test_oracle_minmax_tuned_unif_linear_vs_exact_dtft(Nd, mode):
    """On the reference's self-test set-ups (nufft/newfft.m:599-640):
    'minmax:tuned' (which the self-test runs) within 0.12 % of the exact DTFT;
    'minmax:unif' and 'linear' at Jd = 2 (which it lists and skips as poor)
    within 1 % and 100 %: a wrong phase, Nmid or coefficient set gives errors
    of order 100 % or more (measured: tuned <= 0.08 %, unif <= 0.58 %, linear
    37-85 %, the straw man's own error)."""
    om, x0 = _case(Nd)
    ns = np.zeros(len(Nd))
    Xe = nr.dtft(x0, om, ns)
    xe = nr.dtft_adj(Xe, om, Nd, ns)
    for ktype, Jd, bound in (("minmax:tuned", None, 0.12), ("minmax:unif", None, 1.0),
                             ("linear", (2,) * len(Nd), 100.0)):
        st = nf.newfft_init(om, Nd, Jd=Jd, mode=mode, ktype=ktype)
        assert _mpd(Xe, nf.newfft_for(x0, st)) < bound, ktype
        assert _mpd(xe, nf.newfft_adj(Xe, st)) < bound, ktype


@pytest.mark.parametrize("J,L,alf,m", [(6, 512, 2.34 * 6, 0), (6, 512, 14.0, 1), (8, 256, 18.5, 2),
                                       (4, 1024, 5.0, 3), (6, 512, 3.0, 0)])
def test_kb_user_builders(J, L, alf, m):
    """'kb:user': the KB kernel of order m and its transform (the library's
    series / spherical-Bessel evaluation against scipy's iv / jv)."""
    h = mb.newfft_table("kb:user", 20, J, 40, L, kb_alf=alf, kb_m=m)
    ho = nf.ktype_table("kb:user", 20, J, 40, L, kb_alf=alf, kb_m=m)
    assert np.max(np.abs(h - ho)) <= 1e-13 * np.max(np.abs(ho))
    for N, K in ((20, 40), (21, 32), (64, 128)):
        nmid = np.floor(N / 2)
        s = mb.newfft_scale("kb:user", N, J, K, nmid, kb_alf=alf, kb_m=m)
        so = nf.ktype_scale("kb:user", N, J, K, nmid, kb_alf=alf, kb_m=m)
        assert np.max(np.abs(s - so) / np.abs(so)) <= 1e-12


@pytest.mark.parametrize("alpha,beta", [([1.0], 0.5), ([1, -0.57, 0.14], 0.43), ([1.0], 0.0)])
def test_minmax_user_builders(alpha, beta):
    h = mb.newfft_table("minmax:user", 20, 6, 40, 512, alpha=alpha, beta=beta)
    ho = nf.ktype_table("minmax:user", 20, 6, 40, 512, alpha=alpha, beta=beta)
    assert np.max(np.abs(h - ho)) <= 1e-11 * np.max(np.abs(ho))
    s = mb.newfft_scale("minmax:user", 20, 6, 40, 10.0, alpha=alpha, beta=beta)
    so = nf.ktype_scale("minmax:user", 20, 6, 40, 10.0, alpha=alpha, beta=beta)
    assert np.max(np.abs(s - so) / np.abs(so)) <= 1e-12


@pytest.mark.parametrize("Nd", ND_LIST)
@pytest.mark.parametrize("mode", ["table0", "table1"])
def test_oracle_user_ktypes_vs_exact_dtft(Nd, mode):
    """The self-test's 'kb:user' (kb_m = 0, kb_alf = 2.34 * 6: within the
    'kb:minmax' bounds) and 'minmax:user' (alpha = 1, beta = 0.5, listed and
    skipped as poor: within 1 %), nufft/newfft.m:627-632; 'kb:user' of orders
    1 and 2 (alpha 15, 16) within 1 % (measured <= 0.34 %; scaling factors of
    the wrong order give about 6 %)."""
    om, x0 = _case(Nd)
    dd = len(Nd)
    ns = np.zeros(dd)
    Xe = nr.dtft(x0, om, ns)
    xe = nr.dtft_adj(Xe, om, Nd, ns)
    cases = ((dict(ktype="kb:user", kb_alf=[2.34 * 6] * dd, kb_m=[0] * dd), BOUND[mode]),
             (dict(ktype="kb:user", kb_alf=[15.0] * dd, kb_m=[1] * dd), 1.0),
             (dict(ktype="kb:user", kb_alf=[16.0] * dd, kb_m=[2] * dd), 1.0),
             (dict(ktype="minmax:user", alpha=[[1.0]] * dd, beta=[0.5] * dd), 1.0))
    for kw, bound in cases:
        st = nf.newfft_init(om, Nd, mode=mode, **kw)
        assert _mpd(Xe, nf.newfft_for(x0, st)) < bound, kw
        assert _mpd(xe, nf.newfft_adj(Xe, st)) < bound, kw


def test_user_ktype_errors():
    with pytest.raises(ValueError, match="kb_alf and kb_m required"):
        mb.newfft_table("kb:user", 20, 6, 40, 512, kb_alf=14.0)
    with pytest.raises(ValueError, match="integer"):
        mb.newfft_table("kb:user", 20, 6, 40, 512, kb_alf=14.0, kb_m=0.5)
    with pytest.raises(mb.MirtError, match="alpha >= 0"):
        mb.newfft_scale("kb:user", 20, 6, 40, 10.0, kb_alf=-1.0, kb_m=0)
    with pytest.raises(ValueError, match="alpha/beta"):
        mb.newfft_table("minmax:user", 20, 6, 40, 512, alpha=[1.0])


_COMPLEX_CASES = [("kb:minmax", {}, 20, 6, 40, 512), ("kb:minmax", {}, 21, 6, 32, 256),
                  ("kb:beatty", {}, 20, 6, 40, 512), ("kb:user", dict(kb_alf=15.0, kb_m=1), 20, 6, 40, 512),
                  ("diric", {}, 20, 12, 40, 256), ("linear", {}, 20, 2, 40, 512),
                  ("minmax:kb", {}, 20, 6, 40, 512), ("minmax:kb", {}, 21, 6, 42, 256),
                  ("minmax:unif", {}, 20, 6, 40, 512), ("minmax:tuned", {}, 20, 6, 40, 512),
                  ("minmax:user", dict(alpha=[1.0], beta=0.5), 20, 6, 40, 512)]


@pytest.mark.parametrize("ktype,kw,N,J,K,L", _COMPLEX_CASES)
def test_complex_phasing_table_builders(ktype, kw, N, J, K, L):
    """Every ktype's table with phasing 'complex' (the 'fast' / 'ratio'
    constructions): the library against the oracle."""
    h = mb.newfft_table(ktype, N, J, K, L, phasing="complex", **kw)
    ho = nf.ktype_table_complex(ktype, N, J, K, L, **kw)
    assert np.max(np.abs(h - ho)) <= 1e-11 * np.max(np.abs(ho))
    assert np.max(np.abs(ho.imag)) > 0.1 * np.max(np.abs(ho))


@pytest.mark.parametrize("N,J,K,L", [(20, 6, 40, 512), (21, 6, 42, 1024), (64, 8, 128, 256)])
def test_complex_minmax_kb_table_is_nufft_init_table(N, J, K, L):
    """newfft's 'minmax:kb' with phasing 'complex' (alphas fitted at Nmid =
    (N-1)/2, the phase exp(i gam (N-1)/2 arg)) is nufft_init's min-max:KB
    table -- which the reference's golden vectors pin -- in every entry but
    the last: the 'fast' construction repeats the first entry there
    (newfft_table_init.m:169), nufft_table_init.m writes 0."""
    hn = nf.ktype_table_complex("minmax:kb", N, J, K, L)
    hi = nr.nufft_init_table(np.zeros((1, 1)), (N,), (J,), (K,), (0,), L)["h"][0]
    assert np.array_equal(hn[:-1], hi[:-1])
    assert hn[-1] == hn[0] and hi[-1] == 0


@pytest.mark.parametrize("Nd", ND_LIST + [(6,), (6, 5)])
def test_oracle_complex_phasing_vs_exact_dtft(Nd):
    """Phasing 'complex', mode 'table0' (the self-test's complex runs;
    complex tables are order 0 only): every ktype on the self-test set-ups.
    The table0 lookup of the phase ramp exp(-i pi t (N-1)/K) adds about 0.02 %
    to every kernel (measured: kb:* and 'minmax:tuned' <= 0.11 %, 'minmax:kb'
    <= 0.16 % where its fit is coarse (N = 10, 8; not checked at N = 6, 0.41 %),
    'diric' (Jd = 2 Nd) <= 0.03 %,
    'minmax:unif' / 'minmax:user' <= 0.81 %, 'linear' (Jd = 2) 38-84 %)."""
    om, x0 = _case(Nd)
    dd = len(Nd)
    ns = np.zeros(dd)
    Xe = nr.dtft(x0, om, ns)
    xe = nr.dtft_adj(Xe, om, Nd, ns)
    cases = [("kb:minmax", {}, 0.12), ("kb:beatty", {}, 0.12), ("minmax:tuned", {}, 0.12),
             ("minmax:unif", {}, 1.0), ("linear", dict(Jd=(2,) * dd), 100.0),
             ("kb:user", dict(kb_alf=[2.34 * 6] * dd, kb_m=[0] * dd), 0.12),
             ("minmax:user", dict(alpha=[[1.0]] * dd, beta=[0.5] * dd), 1.0)]
    if 2 * max(Nd) <= 16:
        cases.append(("diric", dict(Jd=tuple(2 * np.asarray(Nd))), 0.12))
    if min(Nd) >= 8:     # below that the reference's fit of the scaling factors has <= 3 terms
        cases.append(("minmax:kb", {}, 0.2))
    for ktype, kw, bound in cases:
        st = nf.newfft_init(om, Nd, mode="table0", phasing="complex", ktype=ktype, **kw)
        assert _mpd(Xe, nf.newfft_for(x0, st)) < bound, ktype
        assert _mpd(xe, nf.newfft_adj(Xe, st)) < bound, ktype


def test_ktype_errors():
    with pytest.raises(ValueError, match="ktype"):
        mb.newfft_table("minmax:other", 20, 6, 40, 512)
    # K = 2 N with a J the tuned tables do not hold
    with pytest.raises(mb.MirtError, match="unknown J,K/N"):
        mb.newfft_table("minmax:tuned", 20, 12, 40, 512)
    lib = mb.load()
    h = np.empty(6 * 8 + 1)
    assert lib.mirt_newfft_ktype_table(7, 20, 6, 40, 8, h.ctypes.data_as(mb._lib._dp)) != 0
    # kb:beatty's shape is not real for a K/N too close to 1/2
    with pytest.raises(mb.MirtError, match="beatty"):
        mb.newfft_table("kb:beatty", 20, 2, 12, 8)


@pytest.mark.parametrize("N,J,K,L", [(20, 6, 40, 512), (21, 6, 42, 2048), (64, 8, 128, 1024),
                                     (10, 5, 20, 256)])
def test_minmax_kb_builders(N, J, K, L):
    """newfft's 'minmax:kb' (phasing 'real', the KB fit at Nmid = floor(N/2)):
    the library's builders against the oracle (the least-squares fit is a QR
    solve in the library and an SVD one in numpy: tables agree to 1e-10)."""
    nmid = np.floor(N / 2)
    h, ho = mb.newfft_table("minmax:kb", N, J, K, L), nf.ktype_table("minmax:kb", N, J, K, L)
    assert np.max(np.abs(h - ho)) <= 1e-10
    s, so = mb.newfft_scale("minmax:kb", N, J, K, nmid), nf.ktype_scale("minmax:kb", N, J, K, nmid)
    assert np.max(np.abs(s - so) / np.abs(so)) <= 1e-12


@pytest.mark.parametrize("Nd", [(21,), (9,), (21, 11)])
def test_minmax_kb_is_nufft_init_interpolator_for_odd_n(Nd):
    """For odd N, floor(N/2) = (N-1)/2: newfft's 'minmax:kb' with phasing 'real'
    uses the same min-max coefficients as nufft_init's 'minmax:kb' (the
    oracle pinned by the reference's golden vectors), only phased differently,
    so the two transforms agree to their tables' quantisation (order 0,
    L = 2^13) -- and both sit at the same distance from the exact DTFT."""
    import oracle
    rng = np.random.default_rng(3)
    D = len(Nd)
    om = 3 * 2 * np.pi * (rng.random((200, D)) - 0.5)
    x0 = rng.random(Nd) + 1j * rng.random(Nd)
    Kd, Jd, Ld = tuple(2 * np.asarray(Nd)), (6,) * D, (2 ** 13,) * D
    so = nf.newfft_init(om, Nd, Jd=Jd, Kd=Kd, mode="table0", Ld=Ld, ktype="minmax:kb")
    Xn = nf.newfft_for(x0, so)
    st = nr.nufft_init_table(om, Nd, Jd, Kd, (0,) * D, Ld)
    Xi = nr.nufft(x0, st, lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"],
                                                          s["Kd"], 0)[:, 0])
    assert np.linalg.norm(Xn - Xi) <= 2e-4 * np.linalg.norm(Xi)
