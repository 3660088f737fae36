"""CPU: nufft_init's interpolators in table mode ('kaiser', 'minmax:kb',
'minmax:tuned', 'minmax:user', 'uniform', 'linear').

* The library's host builders (mirt_nufft_ktype_table / _scale) against the
  oracle's restatement of nufft/nufft_table_init.m:100-116 and
  nufft/nufft_init.m:128-230.
* The oracle's generic construction gives, for 'minmax:kb', exactly the
  nufft_init table and scaling factors that the reference's golden vectors
  pin.
* Every kind within its error of the exact DTFT on the reference's own nufft
  self-test set-up (nufft/nufft.m:10-99: Jd = [5 6], Nd = [60 75], Kd = 2 Nd,
  a 41 x 31 grid of frequencies plus four points), table mode with L = 2^12.
"""
from __future__ import annotations

import numpy as np
import pytest

import mirt_b200 as mb
import oracle
from oracle import nufft_ref as nr

_CASES = [("kaiser", (), 20, 6, 40, 512), ("kaiser", (15.0, 1), 20, 6, 40, 512),
          ("minmax:kb", (), 20, 6, 40, 512), ("minmax:kb", (), 21, 5, 42, 256),
          ("minmax:tuned", (), 20, 6, 40, 512), ("minmax:tuned", (), 20, 5, 40, 256),
          ("minmax:user", ([1.0, -0.57, 0.14], 0.43), 20, 6, 40, 512),
          ("uniform", (), 20, 6, 40, 512), ("linear", (), 20, 2, 40, 512),
          ("linear", (), 21, 3, 42, 256)]


@pytest.mark.parametrize("ktype,params,N,J,K,L", _CASES)
def test_nufft_ktype_builders(ktype, params, N, J, K, L):
    h = mb.nufft_table(ktype, N, J, K, L, *params)
    ho = nr.nufft_ktype_table(ktype, N, J, K, L, *params)
    assert h.shape == (J * L + 1,) and h[-1] == 0
    assert np.max(np.abs(h - ho)) <= 1e-11 * np.max(np.abs(ho))
    s = mb.nufft_scale(ktype, N, J, K, *params)
    so = nr.nufft_ktype_scale(ktype, N, J, K, *params)
    assert np.max(np.abs(s - so) / np.abs(so)) <= 1e-12


@pytest.mark.parametrize("N,J,K,L", [(20, 6, 40, 512), (21, 5, 42, 256), (64, 6, 128, 1024)])
def test_generic_construction_is_the_minmax_kb_table(N, J, K, L):
    """'minmax:kb' through the generic 'fast' construction is bit for bit the
    nufft_init table (and scaling factors) of the pinned oracle."""
    assert np.array_equal(nr.nufft_ktype_table("minmax:kb", N, J, K, L), nr.table_1d(N, J, K, L))
    si = nr.scaling_factors((N,), (J,), (K,)).ravel()
    assert np.array_equal(nr.nufft_ktype_scale("minmax:kb", N, J, K), si)


def _selftest_case():
    Nd, Jd = (60, 75), (5, 6)
    Kd = tuple(2 * np.asarray(Nd))
    gam = 2 * np.pi / np.asarray(Kd)
    o1, o2 = np.meshgrid(np.linspace(-3 * gam[0], 3 * gam[0], 41),
                         np.linspace(-2 * gam[1], gam[1], 31), indexing="ij")
    om = np.stack([np.concatenate([o1.ravel(order="F"), [0, 7.2, 2.6, 3.3]]),
                   np.concatenate([o2.ravel(order="F"), [0, 4.2, -1., 5.5]])], 1)
    x = np.random.default_rng(0).standard_normal(Nd)
    return om, Nd, Jd, Kd, x


@pytest.mark.parametrize("ktype,params,bound", [
    ("minmax:kb", (), 0.05), ("kaiser", (), 0.05), ("minmax:tuned", (), 0.1),
    ("kaiser", ([2.34 * 6 + 0.1] * 2, [0, 0]), 0.25), ("kaiser", ([15.0] * 2, [1, 1]), 0.5),
    ("minmax:user", ([[1.0], [1.0]], [0.5, 0.5]), 1.0), ("uniform", (), 1.0),
    ("linear", (), 15.0)])
def test_oracle_nufft_ktypes_vs_exact_dtft(ktype, params, bound):
    """Max percent difference from the exact DTFT (measured: 0.026 % minmax:kb,
    0.025 % kaiser, 0.05 % minmax:tuned, 0.12 / 0.29 % kaiser with alpha + 0.1 /
    order 1, 0.56 % minmax:user (alpha 1, beta 0.5, the self-test's) and
    uniform, 9.2 % linear).  'linear''s conjugated complex factors change
    nothing measurable here; they are pinned by the two restatements agreeing."""
    om, Nd, Jd, Kd, x = _selftest_case()
    Yd = nr.dtft(x, om, np.zeros(2))
    st = nr.nufft_init_table_ktype(om, Nd, Jd, Kd, np.zeros(2), 2 ** 12, ktype, *params)
    fw = lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0)[:, 0]
    Y = nr.nufft(x, st, fw)
    assert 100 * np.max(np.abs(Y - Yd)) / np.max(np.abs(Yd)) < bound


def test_nufft_init_argument_errors():
    """nufft_init's own checks (nufft_init.m:152-199, nufft_table_init.m:86-97),
    on the host before any device work."""
    om = np.zeros((4, 2))
    with pytest.raises(ValueError, match="identical interpolator"):
        mb.nufft_init(om, (16, 16), (6, 6), (32, 32), (0, 0), "table", 512, "kaiser",
                      [14.0, 15.0], [0, 0])
    with pytest.raises(ValueError, match="both alpha and m"):
        mb.nufft_init(om, (16, 16), (6, 6), (32, 32), (0, 0), "table", 512, "kaiser", [14.0, 14.0])
    with pytest.raises(ValueError, match="alpha/beta"):
        mb.nufft_init(om, (16, 16), (6, 6), (32, 32), (0, 0), "table", 512, "minmax:user")
    with pytest.raises(ValueError, match="unknown kernel type"):
        mb.nufft_init(om, (16, 16), (6, 6), (32, 32), (0, 0), "table", 512, "kb:beatty")
    with pytest.raises(mb.MirtError, match="unknown J,K/N"):
        mb.nufft_table("minmax:tuned", 16, 12, 32, 64)


@pytest.mark.parametrize("ktype,params", [("kaiser", ()), ("kaiser", ([15.0, 15.0], [1, 1])),
                                          ("minmax:tuned", ()), ("uniform", ()), ("linear", ())])
def test_nufft_init_host_tables_match_oracle_st(ktype, params):
    """The host part of mb.nufft_init for these interpolators (the tables and
    st.sn handed to the device plan), on the set-up of the GPU test
    test_nufft_init_other_interpolators, against the oracle's st."""
    Nd, Jd, Kd = (32, 24), (6, 5), (64, 48)
    om = np.random.default_rng(17).uniform(-np.pi, np.pi, (600, 2))
    tables, sn = _nufft_mod().nufft_init_tables(ktype, Nd, Jd, Kd, 2 ** 10, *params)
    so = nr.nufft_init_table_ktype(om, Nd, Jd, Kd, np.zeros(2), 2 ** 10, ktype, *params)
    for d in range(2):
        assert np.max(np.abs(tables[d] - so["h"][d])) <= 1e-11 * np.max(np.abs(so["h"][d]))
    sno = so["sn"].ravel(order="F")
    assert np.max(np.abs(sn - sno)) <= 1e-12 * np.max(np.abs(sno))


def _nufft_mod():
    import importlib
    return importlib.import_module("mirt_b200.nufft")


@pytest.mark.parametrize("ktype,kw", [("kb:minmax", {}), ("minmax:kb", {}), ("minmax:tuned", {}),
                                      ("kb:user", dict(kb_alf=15.0, kb_m=1)),
                                      ("minmax:user", dict(alpha=[1.0, -0.57, 0.14], beta=0.43))])
@pytest.mark.parametrize("Nd", [(20,), (20, 10)])
@pytest.mark.parametrize("phasing", ["real", "complex"])
def test_newfft_host_tables_match_oracle_st(ktype, kw, Nd, phasing):
    """The host part of mb.newfft (tables and st.sn with per-dimension user
    parameters), on the set-ups of the GPU tests test_user_interpolators and
    test_complex_phasing_builtin_tables, against the oracle's st."""
    from oracle import newfft_ref as nf
    dd = len(Nd)
    per_dim = {k: [v] * dd for k, v in kw.items()}
    Jd, Kd = (6,) * dd, tuple(2 * np.asarray(Nd))
    Ld = (2 ** 11,) * dd
    om = np.zeros((3, dd))
    tables, sn = _nufft_mod().newfft_tables(ktype, Nd, Jd, Kd, Ld, phasing, **per_dim)
    so = nf.newfft_init(om, Nd, Jd=Jd, Kd=Kd, mode="table0", Ld=Ld, phasing=phasing,
                        ktype=ktype, **per_dim)
    for d in range(dd):
        assert np.max(np.abs(tables[d] - so["h"][d])) <= 1e-11 * np.max(np.abs(so["h"][d]))
    sno = so["sn"].ravel(order="F")
    assert np.max(np.abs(sn - sno)) <= 1e-11 * np.max(np.abs(sno))
