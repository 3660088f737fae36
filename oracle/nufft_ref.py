"""FP64 numpy restatement of MIRT's table-based NUFFT glue.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py import this module, as the checker.  The product
(mirt_b200) builds its own tables in C++ and never calls into oracle/.

What is restated, with the reference lines followed:

* ``nufft_alpha_kb_fit``  nufft/nufft_alpha_kb_fit.m:13-54 (LS fit of the
  Fourier-series scaling coefficients to the optimised KB scaling factors)
* ``kaiser_bessel_ft``    nufft/kaiser_bessel_ft.m:70-73; the KB shape comes
  from nufft/kaiser_bessel.m:119-140 and nufft/param-data/kaiser,m=0.mat
* ``nufft_scale1``        nufft/nufft_scale.m:54-75
* ``nufft_T``             nufft/private/nufft_T.m:45-75 (tol = 0 -> inv)
* ``nufft_r``             nufft/private/nufft_r.m:32-50
* ``nufft_offset``        nufft/private/nufft_offset.m:18-19
* ``nufft_sinc/diric``    nufft/nufft_sinc.m, nufft/nufft_diric.m:38-40
* ``table_1d``            nufft/nufft_table_init.m:111-134 with the
  interpolator of nufft/nufft_init.m:234-263,287-288
* ``nufft_init_table``    nufft/nufft_table_init.m:38-50 and the sn outer
  product nufft/nufft_init.m:214-232
* ``nufft`` / ``nufft_adj``  nufft/nufft.m:128-165, nufft/nufft_adj.m:32-80,
  nufft/nufft_table_interp.m:35-80, nufft/nufft_table_adj.m:34-76
* ``dtft`` / ``dtft_adj``  nufft/dtft.m:80-112, nufft/dtft_adj.m:40-60

Third-party arithmetic the reference takes from MATLAB built-ins (mldivide,
inv, besselj, besseli, fftn/ifftn; MATLAB is not vendored and no version is
pinned) is replaced by numpy.linalg.lstsq / inv, scipy.special.jv / iv and
numpy.fft.  Arrays use the reference's index order (n1 fastest when
flattened with order='F').
"""
from __future__ import annotations

import numpy as np
from scipy import special

# nufft/param-data/kaiser,m=0.mat: Jlist = 2..16 and abest.zn, the optimised
# KB shape per unit J (alpha = J * zn) for K/N = 2.  Values must match the
# reference's data file for the sn / table parity.
KB_ZN = {2: 2.5, 3: 2.27, 4: 2.31, 5: 2.34, 6: 2.32, 7: 2.32, 8: 2.35, 9: 2.34,
         10: 2.34, 11: 2.35, 12: 2.34, 13: 2.35, 14: 2.35, 15: 2.35, 16: 2.33}


def kb_params_best(J: int, K_N: float) -> tuple[float, float]:
    """(alpha, kb_m) for kaiser_bessel(..., 'best', 0, K_N); kaiser_bessel.m:119-140."""
    if K_N != 2:
        return 2.34 * J, 0.0
    if J in KB_ZN:
        zn = KB_ZN[J]
    else:  # nearest tabulated J (imin(abs(J - Jlist)))
        jl = sorted(KB_ZN)
        zn = KB_ZN[jl[int(np.argmin([abs(J - j) for j in jl]))]]
    return J * zn, 0.0


def kaiser_bessel_ft(u, J, alpha, kb_m=0.0, d=1):
    """Fourier transform of the generalised KB function; kaiser_bessel_ft.m:70-73."""
    u = np.asarray(u, dtype=np.float64)
    z = np.sqrt((2 * np.pi * (J / 2) * u) ** 2 - alpha ** 2 + 0j)
    nu = d / 2 + kb_m
    y = ((2 * np.pi) ** (d / 2) * (J / 2) ** d * alpha ** kb_m / special.iv(kb_m, alpha)
         * special.jv(nu, z) / z ** nu)
    return np.real(y)


def nufft_alpha_kb_fit(N: int, J: int, K: int, Nmid=None):
    """LS fit of Fourier-series scaling coefficients; nufft_alpha_kb_fit.m:13-54
    (its 'Nmid' option; default (N - 1) / 2)."""
    beta = 1.0
    Nmid = (N - 1) / 2 if Nmid is None else Nmid
    L = 13 if N > 40 else int(np.ceil(N / 3))
    nlist = np.arange(N, dtype=np.float64) - Nmid
    kb_a, kb_m = kb_params_best(J, K / N)
    # kaiser_bessel_ft('inline', ...) formats alpha with %g (6 significant digits)
    kb_a = float('%g' % kb_a)
    kb_m = float('%g' % kb_m)
    sn_kaiser = 1.0 / kaiser_bessel_ft(nlist / K, J, kb_a, kb_m, 1)
    gam = 2 * np.pi / K
    X = np.cos((beta * gam * nlist)[:, None] * np.arange(L + 1, dtype=np.float64)[None, :])
    coef, *_ = np.linalg.lstsq(X, sn_kaiser, rcond=None)
    alphas = np.concatenate([[np.real(coef[0])], coef[1:] / 2])
    return alphas, beta


def nufft_scale1(N, K, alpha, beta, Nmid=None):
    """1D scaling factors from Fourier-series coefficients; nufft_scale.m:54-75."""
    if Nmid is None:
        Nmid = (N - 1) / 2
    L = len(alpha) - 1
    n = np.arange(N, dtype=np.float64)
    if L == 0:
        return alpha[0] * np.ones(N, dtype=np.complex128)
    i_gam_n_n0 = 1j * (2 * np.pi / K) * (n - Nmid) * beta
    sn = np.zeros(N, dtype=np.complex128)
    for l1 in range(-L, L + 1):
        alf = alpha[abs(l1)]
        if l1 < 0:
            alf = np.conj(alf)
        sn = sn + alf * np.exp(i_gam_n_n0 * l1)
    return sn


def nufft_sinc(x):
    x = np.asarray(x, dtype=np.float64)
    y = np.ones_like(x)
    nz = x != 0
    y[nz] = np.sin(np.pi * x[nz]) / (np.pi * x[nz])
    return y


def nufft_diric(k, N, K):
    """sinc version of the Dirichlet kernel (use_true_diric = false); nufft_diric.m:38-40."""
    return nufft_sinc(np.asarray(k) / (K / N))


def nufft_T(N, J, K, alpha, beta):
    """T = inv(C'SS'C); nufft_T.m:45-75 with tol = 0 (plain inverse)."""
    L = len(alpha) - 1
    j1, j2 = np.meshgrid(np.arange(1, J + 1), np.arange(1, J + 1), indexing='ij')
    cssc = np.zeros((J, J), dtype=np.complex128)
    for l1 in range(-L, L + 1):
        for l2 in range(-L, L + 1):
            alf1 = alpha[abs(l1)]
            if l1 < 0:
                alf1 = np.conj(alf1)
            alf2 = alpha[abs(l2)]
            if l2 < 0:
                alf2 = np.conj(alf2)
            tmp = j2 - j1 + beta * (l1 - l2)
            cssc = cssc + alf1 * np.conj(alf2) * nufft_diric(tmp, N, K)
    return np.linalg.inv(cssc)


def nufft_offset(om, J, K):
    gam = 2 * np.pi / K
    return np.floor(om / gam - J / 2)


def nufft_r(om, N, J, K, alpha, beta):
    """r vectors and diric arguments, [J, M]; nufft_r.m:32-50."""
    gam = 2 * np.pi / K
    dk = om / gam - nufft_offset(om, J, K)
    arg = -np.arange(1, J + 1, dtype=np.float64)[:, None] + dk[None, :]
    L = len(alpha) - 1
    rr = np.zeros(arg.shape, dtype=np.complex128)
    for l1 in range(-L, L + 1):
        alf = alpha[abs(l1)]
        if l1 < 0:
            alf = np.conj(alf)
        rr = rr + alf * nufft_diric(arg + l1 * beta, N, K)
    return rr, arg


def minmax_interp_1d(om, N, J, K):
    """Per-dimension min-max interpolation coefficients of nufft_init.m:234-263.

    Returns (ud [J, M] complex, kd [J, M] 0-based grid columns)."""
    alpha, beta = nufft_alpha_kb_fit(N, J, K)
    T = nufft_T(N, J, K, alpha, beta)
    r, arg = nufft_r(om, N, J, K, alpha, beta)
    c = T @ r
    gam = 2 * np.pi / K
    phase_scale = 1j * gam * (N - 1) / 2
    ud = np.exp(phase_scale * arg) * c
    koff = nufft_offset(om, J, K)
    kd = np.mod(np.arange(1, J + 1)[:, None] + koff[None, :], K).astype(np.int64)
    return ud, kd


def table_1d(N: int, J: int, K: int, L: int) -> np.ndarray:
    """Complex min-max:KB table of length J*L+1; nufft_table_init.m:111-134."""
    t1 = (J / 2 - 1) + np.arange(L, dtype=np.float64) / L
    om1 = t1 * 2 * np.pi / K
    ud, kd = minmax_interp_1d(om1, N, J, K)
    # 1D sparse matrix p [L, K] with p(m, kd(j, m)) = conj(ud(j, m)) (n_shift = 0,
    # nufft_init.m:287-292); duplicates add as in sparse()
    uu = np.conj(ud)
    p = np.zeros((L, K), dtype=np.complex128)
    for j in range(J):
        np.add.at(p, (np.arange(L), kd[j]), uu[j])
    h = np.concatenate([p[:, jj] for jj in range(J - 1, -1, -1)] + [np.zeros(1)])
    return h


def scaling_factors(Nd, Jd, Kd) -> np.ndarray:
    """sn [(Nd)] as the outer product of conj(1D factors); nufft_init.m:214-232."""
    sn = np.ones(1, dtype=np.complex128)
    for N, J, K in zip(Nd, Jd, Kd):
        alpha, beta = nufft_alpha_kb_fit(N, J, K)
        tmp = nufft_scale1(N, K, alpha, beta)
        sn = np.outer(sn.ravel(order='F'), np.conj(tmp))
    return sn.reshape(tuple(Nd), order='F')


def nufft_init_table(om, Nd, Jd, Kd, n_shift, Ld) -> dict:
    """st = nufft_init(om, Nd, Jd, Kd, n_shift, 'table', Ld, 'minmax:kb')."""
    om = np.asarray(om, dtype=np.float64)
    if om.ndim == 1:
        om = om[:, None]
    dd = len(Nd)
    Ld = list(Ld) if np.ndim(Ld) else [int(Ld)] * dd
    st = dict(om=om, Nd=tuple(Nd), Jd=tuple(Jd), Kd=tuple(Kd), Ld=tuple(Ld),
              n_shift=np.asarray(n_shift, dtype=np.float64), M=om.shape[0])
    st['sn'] = scaling_factors(Nd, Jd, Kd)
    st['h'] = [table_1d(Nd[d], Jd[d], Kd[d], Ld[d]) for d in range(dd)]
    if np.any(st['n_shift'] != 0):
        st['phase_shift'] = np.exp(1j * (om @ st['n_shift']))
    else:
        st['phase_shift'] = None
    st['tm'] = np.stack([om[:, d] / (2 * np.pi / Kd[d]) for d in range(dd)], axis=1)
    return st


def nufft_ktype_table(ktype, N, J, K, L, *params):
    """1D table of nufft_init(..., 'table', L, ktype, params...): nufft_init's
    sparse interpolator (entries conj(exp(i gam (N-1)/2 arg) c),
    nufft_init.m:262-290) read at t1 = J/2 - 1 + l/L by the 'fast'
    construction of nufft_table_init.m:100-116, the last entry 0.  'kaiser'
    [alpha, m]: the KB kernel (alpha 2.34 J, m 0 by default; both printed with
    %g into the inline kernel); 'linear'; the min-max kinds 'minmax:kb',
    'minmax:tuned', 'minmax:user' (alpha list, beta), 'uniform'."""
    from oracle import newfft_ref as nf
    if ktype == "kaiser":
        a, m = params if params else (2.34 * J, 0)
        a, m = float(f"{a:g}"), float(f"{m:g}")

        def coef(arg):
            out = np.zeros_like(arg)
            inside = np.abs(arg) < J / 2
            f = np.sqrt(1 - (arg[inside] / (J / 2)) ** 2)
            out[inside] = f ** m * special.iv(abs(m), a * f) / special.iv(abs(m), a)
            return out
    elif ktype == "linear":
        coef = lambda arg: (1 - np.abs(arg / (J / 2))) * (np.abs(arg) < J / 2)
    else:
        al, b = _nufft_minmax_params(ktype, N, J, K, params)
        T = nufft_T(N, J, K, al, b)

        def coef(arg):
            r = np.zeros(arg.shape)
            for l1 in range(-(len(al) - 1), len(al)):
                r = r + al[abs(l1)] * nufft_diric(arg + l1 * b, N, K)
            return np.real(T @ r)
    h = nf._fast_table_complex(N, J, K, L, coef)
    h[-1] = 0
    return h


def _nufft_minmax_params(ktype, N, J, K, params):
    from oracle import newfft_ref as nf
    if ktype == "minmax:kb":
        return nufft_alpha_kb_fit(N, J, K)
    if ktype == "minmax:tuned":
        return nf.best_alpha(J, N, K)
    if ktype == "minmax:user":
        return np.atleast_1d(np.asarray(params[0], dtype=np.float64)), float(params[1])
    if ktype == "uniform":
        return np.array([1.0]), 0.0
    raise ValueError(ktype)


def nufft_ktype_scale(ktype, N, J, K, *params):
    """The 1D factors of nufft_init's st.sn (conj, as st.sn(:) * tmp' makes
    them; nufft_init.m:210-230): 1 / kaiser_bessel_ft((n - (N-1)/2) / K) for
    'kaiser', nufft_scale for the min-max kinds, 1 / nufft_interp_zn(0, ...)
    (nufft/private/nufft_interp_zn.m) for 'linear'."""
    nc = np.arange(N) - (N - 1) / 2
    if ktype == "kaiser":
        a, m = params if params else (2.34 * J, 0)
        tmp = 1.0 / kaiser_bessel_ft(nc / K, J, a, float(m), 1)
    elif ktype == "linear":
        jlist = np.arange(-J // 2 + 1, J // 2 + 1) if J % 2 == 0 else np.arange(-(J - 1) // 2, (J - 1) // 2 + 1)
        jarg = -jlist[None, :].astype(np.float64)
        F = (1 - np.abs(jarg / (J / 2))) * (np.abs(jarg) < J / 2)
        zn = np.sum(F * np.exp(1j * (2 * np.pi / K) * jarg * nc[:, None]), axis=1)
        tmp = 1.0 / zn
    else:
        al, b = _nufft_minmax_params(ktype, N, J, K, params)
        tmp = nufft_scale1(N, K, al, b)
    return np.conj(tmp)


def nufft_init_table_ktype(om, Nd, Jd, Kd, n_shift, Ld, ktype, *params) -> dict:
    """st = nufft_init(om, Nd, Jd, Kd, n_shift, 'table', Ld, ktype, params...);
    per-dimension params ('kaiser': alpha_list, m_list; 'minmax:user':
    alpha_list, beta_list)."""
    st = nufft_init_table(om, Nd, Jd, Kd, n_shift, Ld)
    dd = len(Nd)
    pd = [tuple(p[d] for p in params) for d in range(dd)] if params else [()] * dd
    st["h"] = [nufft_ktype_table(ktype, Nd[d], Jd[d], Kd[d], st["Ld"][d], *pd[d])
               for d in range(dd)]
    sn = np.ones(1, dtype=np.complex128)
    for d in range(dd):
        sn = np.outer(sn.ravel(order='F'), nufft_ktype_scale(ktype, Nd[d], Jd[d], Kd[d], *pd[d]))
    st["sn"] = sn.reshape(tuple(Nd), order='F')
    return st


def nufft(x, st, interp):
    """X = nufft(x, st); ``interp(Xk_flat_F, st) -> X [M]`` supplies the table gather."""
    Nd, Kd = st['Nd'], st['Kd']
    x = np.asarray(x, dtype=np.complex128).reshape(Nd, order='F') * st['sn']
    Xk = np.fft.fftn(x, s=Kd, axes=tuple(range(len(Kd))))
    X = interp(Xk.ravel(order='F'), st)
    if st['phase_shift'] is not None:
        X = X * st['phase_shift']
    return X


def nufft_adj(X, st, interp_adj):
    """x = nufft_adj(X, st); ``interp_adj(X, st) -> Xk_flat_F [prod(Kd)]``."""
    Nd, Kd = st['Nd'], st['Kd']
    X = np.asarray(X, dtype=np.complex128)
    if st['phase_shift'] is not None:
        X = X * np.conj(st['phase_shift'])
    Xk = interp_adj(X, st).reshape(Kd, order='F')
    x = np.fft.ifftn(Xk, norm='forward')
    x = x[tuple(slice(0, n) for n in Nd)]
    return x * np.conj(st['sn'])


def _dtft_phases(om, Nd, n_shift):
    return [np.exp(-1j * om[:, d][:, None] * (np.arange(Nd[d]) - n_shift[d])[None, :])
            for d in range(len(Nd))]


def dtft(x, om, n_shift, chunk=2048):
    """Exact X(om_m) = sum_n x[n] exp(-i om_m . (n - n_shift)); dtft.m:80-112."""
    om = np.atleast_2d(np.asarray(om, dtype=np.float64))
    if om.shape[0] == 1 and om.shape[1] != len(np.shape(x)):
        om = om.T
    Nd = np.shape(x)
    x = np.asarray(x, dtype=np.complex128)
    out = np.empty(om.shape[0], dtype=np.complex128)
    for s in range(0, om.shape[0], chunk):
        E = _dtft_phases(om[s:s + chunk], Nd, n_shift)
        if len(Nd) == 1:
            out[s:s + chunk] = E[0] @ x
        elif len(Nd) == 2:
            out[s:s + chunk] = np.einsum('ma,mb,ab->m', E[0], E[1], x, optimize=True)
        else:
            y = E[0] @ x.reshape(Nd[0], -1)               # [m, n2*n3]
            y = y.reshape(-1, Nd[1], Nd[2])
            out[s:s + chunk] = np.einsum('mbc,mb,mc->m', y, E[1], E[2], optimize=True)
    return out


def dtft_adj(X, om, Nd, n_shift, chunk=2048):
    """Exact adjoint x[n] = sum_m X_m exp(+i om_m . (n - n_shift)); dtft_adj.m:40-60."""
    om = np.asarray(om, dtype=np.float64)
    if om.ndim == 1:
        om = om[:, None]
    X = np.asarray(X, dtype=np.complex128)
    x = np.zeros(Nd, dtype=np.complex128)
    for s in range(0, om.shape[0], chunk):
        E = [np.conj(e) for e in _dtft_phases(om[s:s + chunk], Nd, n_shift)]
        w = X[s:s + chunk]
        if len(Nd) == 1:
            x += w @ E[0]
        elif len(Nd) == 2:
            x += np.einsum('m,ma,mb->ab', w, E[0], E[1], optimize=True)
        else:
            # separable: x[a, b, c] += sum_m E0[m, a] (w_m E1[m, b] E2[m, c]) as one matmul
            B = (w[:, None] * E[1])[:, :, None] * E[2][:, None, :]
            x += (E[0].T @ B.reshape(len(w), -1)).reshape(Nd)
    return x
