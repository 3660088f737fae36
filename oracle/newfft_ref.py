"""FP64 numpy restatement of MIRT's newfft in table mode (real KB kernel).

TEST INFRASTRUCTURE ONLY.  Only tests/ and ``__graft_entry__.smoke()`` import
this module, as the checker.  The product (mirt_b200) builds its own tables in
C++ and never calls into oracle/.

What is restated, with the reference lines followed:

* ``Nmid``               nufft/newfft.m:146-151 (floor(N/2) for phasing 'real',
  (N-1)/2 otherwise)
* ``kb_table``           the 'ratio' table of nufft/private/newfft_table_init.m:
  140-184 for ktype 'kb:minmax' (kernel nufft/kaiser_bessel.m:68-69,106-117 with
  alpha = 2.34 J, kb_m = 0; the inline kernel string prints alpha with %g,
  nufft/kaiser_bessel.m:80-82).  The table reads the sparse interpolator of a
  fake N = J problem column by column (J:-1:1), which for a kernel of the
  offset alone is the kernel sampled at t = -J/2 + i/L; the last entry
  repeats the first (0 at |t| = J/2).
* ``kb_scale``           1 / kaiser_bessel_ft((n - Nmid) / K, J, alpha, 0, 1),
  nufft/newfft.m:352-356, outer product nufft/newfft.m:366-375
* ``beatty_alpha``       ktype 'kb:beatty': pi sqrt(J^2 / r^2 (r - 1/2)^2 - 0.8),
  r = K / N, kb_m = 0 (nufft/newfft.m:275-283); its table and scale are
  ``kb_table`` / ``kb_scale`` with that alpha
* ``minmax_kb_table``    ktype 'minmax:kb' with phasing 'real' (nufft/newfft.m:315-320,
  384-395): alphas / beta of nufft_alpha_kb_fit at Nmid = floor(N/2), c = T r
  (nufft/private/nufft_T.m, nufft_r.m) without phase, read by the 'fast'
  construction; scale the real part of nufft_scale1 at Nmid
* ``diric_table``        ktype 'diric' with phasing 'real' (nufft/newfft.m:256-266):
  N' / K nufft_diric(t, N', K, true) with N' = 2 floor((K + 1) / 2) - 1
  (nufft/nufft_diric.m:31-36), read by the 'fast' construction of
  nufft/private/newfft_table_init.m:160-169 through nufft/private/nufft_coef.m
  (the kernel at t = -J/2 + i/L, i < J L; the last entry repeats the first);
  its scaling factors are 1 (nufft/newfft.m:354-355)
* ``minmax_table``       ktypes 'minmax:unif' (alpha = 1, beta = 0,
  nufft/newfft.m:337-341) and 'minmax:tuned' (``best_alpha``: nufft_best_alpha(J,
  0, K/N), nufft/newfft.m:322-327), the 'minmax:kb' construction with those
  coefficients; scale the real part of nufft_scale1
* ``linear_table``       ktype 'linear' (nufft/newfft.m:268-273), the triangle
  read by the 'fast' construction; ``linear_scale`` newfft_scale_tri
  (nufft/newfft.m:535-550), evaluated per dimension
* ``kb_table(J, L, alpha, kb_m)`` / ``kb_scale``  ktype 'kb:user' (nufft/newfft.m:300-313):
  the KB kernel of order kb_m, its transform nufft/kaiser_bessel_ft.m:70-73
* ``minmax_table`` with the caller's alpha / beta: ktype 'minmax:user'
  (nufft/newfft.m:329-335)
* ``ktype_table_complex`` every ktype with phasing 'complex': the sparse
  interpolator's entries conj(exp(i gam (N-1)/2 arg) c) (nufft/newfft.m:405-411,
  446) read by the 'fast' construction, or for 'kb:*' by the 'ratio' one with
  its phase correction (nufft/private/newfft_table_init.m:160-184)
* ``phase_before``       nufft/newfft.m:511-520
* ``phase_after``        nufft/newfft.m:522-527
* ``newfft_for/adj``     nufft/private/newfft_approx_for.m:15-63,
  nufft/private/newfft_approx_adj.m:30-82, the interpolation through the
  table kernels of oracle/interp_table.c (st.order from
  nufft/private/newfft_table_init.m:40-49: 0 for 'table0' with L = 2^11,
  1 for 'table1' with L = 2^9; phase_shift empty, :34).

scipy.special.iv stands in for MATLAB's besseli.
"""
from __future__ import annotations

import numpy as np
from scipy import special

import oracle
from oracle import nufft_ref as nr


def nmid_of(Nd, phasing="real"):
    Nd = np.asarray(Nd, dtype=np.float64)
    return np.floor(Nd / 2) if phasing == "real" else (Nd - 1) / 2


def kb_alpha(J):
    return 2.34 * J


def beatty_alpha(N, J, K):
    r = K / N
    return np.pi * np.sqrt(J ** 2 / r ** 2 * (r - 0.5) ** 2 - 0.8)


def diric_table(J: int, K: int, L: int) -> np.ndarray:
    """Real [J*L+1] table of ktype 'diric' with phasing 'real'."""
    Np = 2 * ((K + 1) // 2) - 1
    k = -J / 2 + np.arange(J * L) / L
    t = np.pi / K * k
    f = np.sin(t)
    big = np.abs(f) > 1e-12
    out = np.sign(np.cos(t * (Np - 1)))
    out[big] = np.sin(Np * t[big]) / (Np * f[big])
    h = Np / K * out
    return np.append(h, h[0])


def kb_table(J: int, L: int, alpha=None, kb_m=0) -> np.ndarray:
    """Real [J*L+1] table of the KB kernel of shape alpha (default 2.34 J:
    'kb:minmax') and order kb_m, f^m I_m(alpha f) / I_m(alpha)
    (nufft/kaiser_bessel.m:106-117), alpha and kb_m printed with %g as the
    inline kernel does (:80-82)."""
    alpha = float(f"{(kb_alpha(J) if alpha is None else alpha):g}")
    kb_m = float(f"{kb_m:g}")
    t = (np.arange(J * L + 1) - J * L / 2) / L
    h = np.zeros(J * L + 1)
    inside = np.abs(t) < J / 2
    f = np.sqrt(1 - (t[inside] / (J / 2)) ** 2)
    h[inside] = f ** kb_m * special.iv(abs(kb_m), alpha * f) / special.iv(abs(kb_m), alpha)
    return h


def kb_scale(N: int, J: int, K: int, Nmid: float, alpha=None, kb_m=0) -> np.ndarray:
    nc = np.arange(N) - Nmid
    return 1.0 / nr.kaiser_bessel_ft(nc / K, J, kb_alpha(J) if alpha is None else alpha,
                                     float(kb_m), 1)


# nufft/nufft_best_alpha.m:13-33: tuned Fourier coefficients of the scaling
# factors for K/N = 2, J -> (alpha_0 .. alpha_L, beta); the L = 3 sets are the
# reference's choice for J = 4 and 6 (its "L = 0: best available", :37-43)
_BEST_ALPHA_L3 = {4: ([1, -0.5319, 0.1522, -0.0199], 0.6339),
                  6: ([1, -0.6903, 0.2138, -0.0191], 0.2254)}
_BEST_ALPHA_L2 = {2: ([1, -0.200, -0.04], 0.34), 3: ([1, -0.485, 0.090], 0.48),
                  4: ([1, -0.470, 0.085], 0.56), 5: ([1, -0.4825, 0.12], 0.495),
                  6: ([1, -0.57, 0.14], 0.43), 7: ([1, -0.465, 0.07], 0.65),
                  8: ([1, -0.540, 0.16], 0.47), 9: ([1, -0.625, 0.14], 0.325),
                  10: ([1, -0.57, 0.185], 0.43)}


def best_alpha(J, N, K):
    """nufft_best_alpha(J, 0, K/N) (nufft/nufft_best_alpha.m:35-77): for K/N = 2
    the L = 3 set where there is one, else the L = 2 set (ValueError for a J
    without one: newfft's 'unknown J,K/N'); for any other K/N alpha = 1,
    beta = 0.5."""
    if K / N != 2:
        return np.array([1.0]), 0.5
    table = _BEST_ALPHA_L3 if J in _BEST_ALPHA_L3 else _BEST_ALPHA_L2
    if J not in table:
        raise ValueError("unknown J,K/N")
    a, b = table[J]
    return np.asarray(a, dtype=np.float64), b


def minmax_table(N, J, K, L, alpha, beta):
    """Real [J*L+1] table of a 'minmax:*' ktype with phasing 'real': the min-max
    coefficients c = T r (no phase) for scaling coefficients alpha, beta read
    by the 'fast' construction, the last entry repeating the first."""
    T = nr.nufft_T(N, J, K, alpha, beta)
    t1 = (J / 2 - 1) + np.arange(L, dtype=np.float64) / L
    om1 = t1 * 2 * np.pi / K
    r, _ = nr.nufft_r(om1, N, J, K, alpha, beta)
    c = np.real(T @ r)
    koff = nr.nufft_offset(om1, J, K)
    kd = np.mod(np.arange(1, J + 1)[:, None] + koff[None, :], K).astype(np.int64)
    p = np.zeros((L, K))
    for j in range(J):
        np.add.at(p, (np.arange(L), kd[j]), c[j])
    h = np.concatenate([p[:, jj] for jj in range(J - 1, -1, -1)])
    return np.append(h, h[0])


def minmax_kb_table(N, J, K, L):
    """ktype 'minmax:kb': the alphas fitted at Nmid = floor(N/2)."""
    alpha, beta = nr.nufft_alpha_kb_fit(N, J, K, Nmid=np.floor(N / 2))
    return minmax_table(N, J, K, L, alpha, beta)


def minmax_kb_scale(N, J, K, Nmid):
    alpha, beta = nr.nufft_alpha_kb_fit(N, J, K, Nmid=Nmid)
    return np.real(nr.nufft_scale1(N, K, alpha, beta, Nmid))


def linear_table(J, L):
    """ktype 'linear' (nufft/newfft.m:268-273): (1 - |t/(J/2)|) (|t| < J/2) at
    t = -J/2 + i/L, i < J L, the last entry repeating the first."""
    t = -J / 2 + np.arange(J * L) / L
    h = (1 - np.abs(t / (J / 2))) * (np.abs(t) < J / 2)
    return np.append(h, h[0])


def linear_scale(N, J, K, Nmid):
    """newfft_scale_tri (nufft/newfft.m:535-550) at one dimension's Nmid."""
    nc = np.arange(N) - Nmid
    fun = lambda x: J * nr.nufft_sinc(J * x / K) ** 2
    tmp = sum(np.abs(fun(nc - ll * K)) ** 2 for ll in range(-3, 4))
    return fun(nc) / tmp


def ktype_table(ktype, N, J, K, L, kb_alf=None, kb_m=None, alpha=None, beta=None):
    if ktype == "kb:user":
        return kb_table(J, L, kb_alf, kb_m)
    if ktype == "minmax:user":
        return minmax_table(N, J, K, L, np.atleast_1d(np.asarray(alpha, dtype=np.float64)), beta)
    if ktype == "kb:minmax":
        return kb_table(J, L)
    if ktype == "kb:beatty":
        return kb_table(J, L, beatty_alpha(N, J, K))
    if ktype == "diric":
        return diric_table(J, K, L)
    if ktype == "minmax:kb":
        return minmax_kb_table(N, J, K, L)
    if ktype == "minmax:unif":
        return minmax_table(N, J, K, L, np.array([1.0]), 0.0)
    if ktype == "minmax:tuned":
        return minmax_table(N, J, K, L, *best_alpha(J, N, K))
    if ktype == "linear":
        return linear_table(J, L)
    raise ValueError(ktype)


def ktype_scale(ktype, N, J, K, Nmid, kb_alf=None, kb_m=None, alpha=None, beta=None):
    if ktype == "kb:user":
        return kb_scale(N, J, K, Nmid, kb_alf, kb_m)
    if ktype == "minmax:user":
        return np.real(nr.nufft_scale1(N, K, np.atleast_1d(np.asarray(alpha, dtype=np.float64)),
                                       beta, Nmid))
    if ktype == "kb:minmax":
        return kb_scale(N, J, K, Nmid)
    if ktype == "kb:beatty":
        return kb_scale(N, J, K, Nmid, beatty_alpha(N, J, K))
    if ktype == "diric":
        return np.ones(N)
    if ktype == "minmax:kb":
        return minmax_kb_scale(N, J, K, Nmid)
    if ktype == "minmax:unif":
        return np.real(nr.nufft_scale1(N, K, np.array([1.0]), 0.0, Nmid))
    if ktype == "minmax:tuned":
        return np.real(nr.nufft_scale1(N, K, *best_alpha(J, N, K), Nmid))
    if ktype == "linear":
        return linear_scale(N, J, K, Nmid)
    raise ValueError(ktype)


def _fast_table_complex(N, J, K, L, coef):
    """The 'fast' construction (nufft/private/newfft_table_init.m:160-169) with
    phasing 'complex': sparse-interpolator entries conj(exp(i gam (N-1)/2 arg)
    c(arg)) (nufft/newfft.m:405-411, 446) at columns mod(koff + j, K), the
    table columns J .. 1, the last entry repeating the first.  K may be
    fractional (the 'ratio' construction's fake problem)."""
    gam = 2 * np.pi / K
    t1 = (J / 2 - 1) + np.arange(L, dtype=np.float64) / L
    om1 = t1 * 2 * np.pi / K
    koff = nr.nufft_offset(om1, J, K)
    dk = om1 / gam - koff
    arg = -np.arange(1, J + 1, dtype=np.float64)[:, None] + dk[None, :]      # [J, L]
    uu = np.conj(np.exp(1j * gam * (N - 1) / 2 * arg) * coef(arg))
    kd = np.mod(np.arange(1, J + 1)[:, None] + koff[None, :], K)
    p = np.zeros((L, J), dtype=np.complex128)
    for j in range(J):
        use = (kd[j] < J) & (kd[j] == np.floor(kd[j]))
        np.add.at(p, (np.arange(L)[use], kd[j][use].astype(np.int64)), uu[j][use])
    h = np.concatenate([p[:, jj] for jj in range(J - 1, -1, -1)])
    return np.append(h, h[0])


def ktype_table_complex(ktype, N, J, K, L, kb_alf=None, kb_m=None, alpha=None, beta=None):
    """Complex [J*L+1] table of `ktype` with phasing 'complex': the 'ratio'
    construction for 'kb:*' (nufft/private/newfft_table_init.m:173-184: fake
    N' = J, K' = J K / N, then exp(i pi t (1/K - 1/K'))), the 'fast' one for
    the others ('diric' with the caller's N: no odd-N trick; 'minmax:kb' fitted
    at Nmid = (N-1)/2)."""
    if ktype.startswith("kb:"):
        if ktype == "kb:minmax":
            a, m = kb_alpha(J), 0
        elif ktype == "kb:beatty":
            a, m = beatty_alpha(N, J, K), 0
        else:
            a, m = kb_alf, kb_m
        a = float(f"{a:g}")
        m = float(f"{m:g}")

        def kern(arg):
            out = np.zeros_like(arg)
            inside = np.abs(arg) < J / 2
            f = np.sqrt(1 - (arg[inside] / (J / 2)) ** 2)
            out[inside] = f ** m * special.iv(abs(m), a * f) / special.iv(abs(m), a)
            return out
        Kf = J * K / N
        h = _fast_table_complex(J, J, Kf, L, kern)
        t0 = (np.arange(J * L + 1) - J * L / 2) / L
        return h * np.exp(1j * np.pi * t0 * (1 / K - 1 / Kf))
    if ktype == "diric":
        def kern(arg):
            t = np.pi / K * arg
            f = np.sin(t)
            big = np.abs(f) > 1e-12
            out = np.sign(np.cos(t * (N - 1)))
            out[big] = np.sin(N * t[big]) / (N * f[big])
            return N / K * out
        return _fast_table_complex(N, J, K, L, kern)
    if ktype == "linear":
        return _fast_table_complex(N, J, K, L,
                                   lambda arg: (1 - np.abs(arg / (J / 2))) * (np.abs(arg) < J / 2))
    if ktype == "minmax:kb":
        al, b = nr.nufft_alpha_kb_fit(N, J, K)
    elif ktype == "minmax:unif":
        al, b = np.array([1.0]), 0.0
    elif ktype == "minmax:tuned":
        al, b = best_alpha(J, N, K)
    elif ktype == "minmax:user":
        al, b = np.atleast_1d(np.asarray(alpha, dtype=np.float64)), beta
    else:
        raise ValueError(ktype)
    T = nr.nufft_T(N, J, K, al, b)

    def coef(arg):
        r = np.zeros(arg.shape)
        L_ = len(al) - 1
        for l1 in range(-L_, L_ + 1):
            r = r + al[abs(l1)] * nr.nufft_diric(arg + l1 * b, N, K)
        return np.real(T @ r)
    return _fast_table_complex(N, J, K, L, coef)


def phase_before(Kd, Nmid) -> np.ndarray:
    """exp(i 2 pi sum_d k_d / K_d Nmid_d) over the grid [(Kd)]."""
    ph = np.zeros(())
    for K, m in zip(Kd, Nmid):
        tmp = 2 * np.pi * np.arange(K) / K * m
        ph = np.add.outer(ph, tmp) if ph.ndim else tmp
    return np.exp(1j * ph)


def newfft_init(om, Nd, Jd=None, Kd=None, n_shift=None, mode="table1", Ld=None,
                phasing="real", h=None, sn=None, ktype="kb:minmax", kb_alf=None, kb_m=None,
                alpha=None, beta=None) -> dict:
    """st of newfft(om, Nd, 'Jd', Jd, 'Kd', Kd, 'n_shift', n_shift, 'mode', mode,
    'oversample', Ld, 'phasing', phasing, 'ktype', ktype[, 'kb_alf', kb_alf,
    'kb_m', kb_m | 'alpha', alpha, 'beta', beta]) for the built-in ktypes (or
    the caller's tables h and scaling factors sn); user parameters are given
    per dimension."""
    om = np.asarray(om, dtype=np.float64)
    if om.ndim == 1:
        om = om[:, None]
    dd = len(Nd)
    Jd = tuple([6] * dd if Jd is None else Jd)
    Kd = tuple(2 * np.asarray(Nd) if Kd is None else Kd)
    n_shift = np.zeros(dd) if n_shift is None else np.asarray(n_shift, dtype=np.float64)
    order = {"table0": 0, "table1": 1}[mode]
    if Ld is None:
        Ld = 2 ** 11 if order == 0 else 2 ** 9
    Ld = tuple(Ld if np.ndim(Ld) else [int(Ld)] * dd)
    Nmid = nmid_of(Nd, phasing)
    def user(d):
        pick = lambda v: None if v is None else v[d]
        return dict(kb_alf=pick(kb_alf), kb_m=pick(kb_m), alpha=pick(alpha), beta=pick(beta))
    if h is None:
        make = ktype_table_complex if phasing == "complex" else ktype_table
        h = [make(ktype, Nd[d], Jd[d], Kd[d], Ld[d], **user(d)) for d in range(dd)]
    if sn is None:
        s = np.ones(1)
        for d in range(dd):
            s = np.outer(s.ravel(order="F"), ktype_scale(ktype, Nd[d], Jd[d], Kd[d], Nmid[d],
                                                         **user(d)))
        sn = s.reshape(tuple(Nd), order="F")
    st = dict(om=om, Nd=tuple(Nd), Jd=Jd, Kd=Kd, Ld=Ld, order=order, Nmid=Nmid,
              n_shift=n_shift, h=h, sn=np.asarray(sn).reshape(tuple(Nd), order="F"),
              tm=np.stack([om[:, d] / (2 * np.pi / Kd[d]) for d in range(dd)], axis=1))
    if phasing in ("real", "flipreal"):
        st["phase_before"] = phase_before(Kd, Nmid)
        st["phase_after"] = np.exp(1j * (om @ (n_shift - Nmid)))
    else:
        st["phase_before"] = None
        st["phase_after"] = None
    return st


def newfft_for(x, st):
    """X = st.fft(x) for one image x [(Nd)]."""
    Nd, Kd = st["Nd"], st["Kd"]
    x = np.asarray(x, dtype=np.complex128).reshape(Nd, order="F") * st["sn"]
    Xk = np.fft.fftn(x, s=Kd, axes=tuple(range(len(Kd))))
    if st["phase_before"] is not None:
        Xk = Xk * st["phase_before"]
    X = oracle.interp_for(Xk.ravel(order="F"), st["h"], st["Jd"], st["Ld"], st["tm"], Kd,
                          st["order"])[:, 0]
    if st["phase_after"] is not None:
        X = X * st["phase_after"]
    return X


def newfft_adj(X, st):
    """x = st.adj(X) for one column X [M]."""
    Nd, Kd = st["Nd"], st["Kd"]
    X = np.asarray(X, dtype=np.complex128)
    if st["phase_after"] is not None:
        X = X * np.conj(st["phase_after"])
    Xk = oracle.interp_adj(X, st["h"], st["Jd"], st["Ld"], st["tm"], Kd,
                           st["order"])[:, 0].reshape(Kd, order="F")
    if st["phase_before"] is not None:
        Xk = Xk * np.conj(st["phase_before"])
    x = np.fft.ifftn(Xk, norm="forward")[tuple(slice(0, n) for n in Nd)]
    return x * np.conj(st["sn"])
