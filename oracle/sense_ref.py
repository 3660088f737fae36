"""FP64 restatement of CG-SENSE: Asense, the quadratic Reg1 penalty and qpwls_pcg1.

TEST INFRASTRUCTURE ONLY (the checker of mirt_sense_*).

* A x = [G (s_c .* x)]_c (systems/Asense.m:53-56) with G the table NUFFT of
  oracle.nufft_ref on the reference's own interpolation kernels;
* R x = C'C x for Reg1's defaults: offsets [1 nx nx+1 nx-1]
  (penalty/penalty_offsets.m), first-order differences, 'tight' edges
  (penalty/Rweights.m:290-300: only pairs with both pixels inside the image)
  and weights beta / |offset| (distance_power 1);
* qpwls_pcg1 (wls/qpwls_pcg1.m:94-189), with precon = 1 or the circulant
  preconditioner of the device solver.
Images are numpy [N2, N1] (n1 fastest, the device layout); data [M, C].
"""
from __future__ import annotations

import numpy as np

import oracle
from oracle import nufft_ref as nr


def _impl():
    return "ref" if oracle.ref_available() else "port"


class Sense64:
    def __init__(self, om, N, K, sens, beta, J=6, L=1024):
        self.st = nr.nufft_init_table(om, (N, N), (J, J), (K, K), (N / 2, N / 2), (L, L))
        self.N, self.K = N, K
        self.sens = np.asarray(sens, dtype=np.complex128)          # [N2, N1, C]
        self.C = self.sens.shape[-1]
        self.beta = float(beta)

    def forward(self, x):
        st = self.st
        xs = self.sens * np.asarray(x, np.complex128)[:, :, None]  # [N2, N1, C]
        cks = []
        for c in range(self.C):
            img = xs[:, :, c].T * st["sn"]                            # [n1, n2]
            cks.append(np.fft.fftn(img, s=st["Kd"], axes=(0, 1)).ravel(order="F"))
        Y = oracle.interp_for(np.stack(cks, 1), st["h"], st["Jd"], st["Ld"], st["tm"], st["Kd"], 0,
                              impl=_impl(), nthreads=8)
        if st["phase_shift"] is not None:
            Y = Y * st["phase_shift"][:, None]
        return Y

    def adjoint(self, Y):
        st = self.st
        Y = np.asarray(Y, np.complex128)
        if st["phase_shift"] is not None:
            Y = Y * np.conj(st["phase_shift"])[:, None]
        ck = oracle.interp_adj(Y, st["h"], st["Jd"], st["Ld"], st["tm"], st["Kd"], 0,
                               impl=_impl(), nthreads=8)
        out = np.zeros((self.N, self.N), np.complex128)
        for c in range(self.C):
            g = np.fft.ifftn(ck[:, c].reshape(st["Kd"], order="F"), norm="forward")
            img = (g[:self.N, :self.N] * np.conj(st["sn"])).T              # [N2, N1]
            out += np.conj(self.sens[:, :, c]) * img
        return out

    def reg(self, x):
        x = np.asarray(x, np.complex128)                           # [N2, N1]
        out = np.zeros_like(x)
        for d1, d2, w in ((1, 0, 1.0), (0, 1, 1.0), (1, 1, 2 ** -0.5), (-1, 1, 2 ** -0.5)):
            w = w * self.beta
            # pairs (n, n - d): rows i2 >= d2, columns with i1 - d1 in range
            n2 = self.N
            a1, b1 = max(d1, 0), n2 + min(d1, 0)
            diff = x[d2:, a1:b1] - x[:n2 - d2, a1 - d1:b1 - d1]
            out[d2:, a1:b1] += w * diff
            out[:n2 - d2, a1 - d1:b1 - d1] -= w * diff
        return out


def circulant_precon(A: Sense64):
    """The circulant preconditioner of the device solver, in FP64: spectrum
    1 / max(lam Re H1 + r, 1e-3 max(lam Re H1)) on the 2N grid, H1 the FFT of
    the Toeplitz embedding of G'G (oracle.toeplitz_ref), lam the mean coil
    power, r the spectrum of the Reg1 penalty; applied as crop(ifft2(Hp
    fft2(pad(x)))).  Returns a function of an image [N2, N1]."""
    from oracle import toeplitz_ref as tr
    st = A.st
    N = A.N
    H = tr.gram_kernel(st["om"], (N, N), st["Kd"], st["Jd"], st["Ld"]).real    # [q1, q2]
    lam = np.mean(np.sum(np.abs(A.sens) ** 2, axis=-1))
    a = np.pi * np.arange(2 * N) / N
    A1, A2 = np.meshgrid(a, a, indexing="ij")
    r = A.beta * ((2 - 2 * np.cos(A1)) + (2 - 2 * np.cos(A2))
                  + ((2 - 2 * np.cos(A1 + A2)) + (2 - 2 * np.cos(A2 - A1))) / np.sqrt(2))
    v = lam * H + r
    Hp = 1.0 / np.maximum(v, 1e-3 * np.max(lam * H))

    def apply(g):
        X = np.zeros((2 * N, 2 * N), np.complex128)
        X[:N, :N] = g.T                                       # [n1, n2]
        return np.fft.ifft2(Hp * np.fft.fft2(X))[:N, :N].T
    return apply


def qpwls_pcg1(x, A: Sense64, W, yi, niter, precon=None):
    """Iterates of wls/qpwls_pcg1.m:94-189 in FP64 (precon: a function of the
    gradient image, or None for 1); returns the list [x_0, x_1, ..., x_niter]."""
    x = np.asarray(x, np.complex128).copy()
    W = 1.0 if W is None else np.asarray(W, np.float64)[:, None]
    Ax = A.forward(x)
    Rx = A.reg(x)
    xs = [x.copy()]
    oldinprod = 0.0
    ddir = None
    for it in range(1, niter + 1):
        ngrad = A.adjoint(W * (yi - Ax)) - Rx
        pregrad = ngrad if precon is None else precon(ngrad)
        newinprod = np.real(np.vdot(ngrad, pregrad))
        if it == 1:
            ddir = pregrad
        else:
            gamma = 0.0 if oldinprod == 0 else newinprod / oldinprod
            ddir = pregrad + gamma * ddir
        oldinprod = newinprod
        Adir = A.forward(ddir)
        Rdir = A.reg(ddir)
        denom = np.real(np.vdot(Adir, W * Adir)) + np.real(np.vdot(ddir, Rdir))
        step = 0.0 if denom == 0 else np.real(np.vdot(ddir, ngrad)) / denom
        Ax = Ax + step * Adir
        Rx = Rx + step * Rdir
        x = x + step * ddir
        xs.append(x.copy())
    return xs
