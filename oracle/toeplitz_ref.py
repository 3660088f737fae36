"""FP64 restatement of the Toeplitz Gram operator (systems/Gnufft_gram.m, 2D).

TEST INFRASTRUCTURE ONLY (the checker of mirt_toeplitz_* and the Gram-form
CG-SENSE).  ``gram_kernel`` follows Gnufft_gram_init2 (:183-198): two
adjoint table NUFFTs of the weights without phase shift (omega and omega with
omega_1 negated, Gnufft_gram_setup2 :261-275), the block layout of the
2N1 x 2N2 circulant, the Hermitian average of dsft_gram_hermitify, and the
FFT; ``gram_apply`` is Gnufft_gram_mult (:339-348).  Arrays are indexed
[n1, n2] here (MATLAB order); the device layout [n2][n1] is the transpose.
"""
from __future__ import annotations

import numpy as np

import oracle
from oracle import nufft_ref as nr


def _impl():
    return "ref" if oracle.ref_available() else "port"


def _adj(om, N, K, J, L, w):
    st = nr.nufft_init_table(om, N, J, K, (0.0, 0.0), L)

    def interp_adj(X, st):
        return oracle.interp_adj(np.asarray(X)[:, None], st["h"], st["Jd"], st["Ld"], st["tm"],
                                 st["Kd"], 0, impl=_impl(), nthreads=8)[:, 0]

    return nr.nufft_adj(np.asarray(w, np.complex128), st, interp_adj)   # [N1, N2]


def gram_kernel(om, N, K, J=(6, 6), L=(1024, 1024), w=None):
    """FFT of the Hermitian circulant kernel, [2N1, 2N2] (index [q1, q2])."""
    om = np.asarray(om, np.float64)
    w = np.ones(len(om)) if w is None else np.asarray(w, np.float64)
    N1, N2 = N
    b1 = _adj(om, N, K, J, L, w)
    om2 = om.copy()
    om2[:, 0] = -om2[:, 0]
    b2 = _adj(om2, N, K, J, L, w)
    kern = np.zeros((2 * N1, 2 * N2), np.complex128)
    kern[:N1, :N2] = b1
    top_right = np.concatenate([b1[:1, 1:], b2[1:, 1:]], 0)            # [N1, N2-1]
    kern[:N1, N2 + 1:] = np.conj(top_right[:, ::-1])
    kern[N1 + 1:, :N2] = b2[1:, :][::-1, :]
    kern[N1 + 1:, N2 + 1:] = np.conj(b1[1:, 1:])[::-1, ::-1]
    m1 = (-np.arange(2 * N1)) % (2 * N1)
    m2 = (-np.arange(2 * N2)) % (2 * N2)
    kern = (kern + np.conj(kern[np.ix_(m1, m2)])) / 2
    return np.fft.fft2(kern)


def gram_apply(H, x):
    """crop(ifft2(H fft2(pad(x)))) for x [N1, N2]."""
    N1, N2 = H.shape[0] // 2, H.shape[1] // 2
    X = np.zeros(H.shape, np.complex128)
    X[:N1, :N2] = x
    return np.fft.ifft2(H * np.fft.fft2(X))[:N1, :N2]


def gram_exact(om, N, x, w=None):
    """sum_m w_m e(omega_m) e(omega_m)^H x with the exact DTFT (small cases)."""
    om = np.asarray(om, np.float64)
    w = np.ones(len(om)) if w is None else np.asarray(w)
    n1, n2 = np.meshgrid(np.arange(N[0]), np.arange(N[1]), indexing="ij")
    E = np.exp(-1j * (np.outer(om[:, 0], n1.ravel()) + np.outer(om[:, 1], n2.ravel())))
    return (E.conj().T @ (w * (E @ x.ravel()))).reshape(N)
