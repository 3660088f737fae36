"""Batched CG-SENSE on the device NUFFT: Asense + Reg1 + qpwls_pcg1.

Mirrors the reference's pieces: ``Asense(G, sens)`` (systems/Asense.m), the
quadratic ``Reg1`` penalty with its default offsets and 'tight' edges
(penalty/Reg1.m, penalty/Rweights.m) and ``qpwls_pcg1`` (wls/qpwls_pcg1.m,
precon = 1).  One NUFFT plan carries a batch of problems of the same image
size and coil count (one slice per problem); every problem keeps its own CG
scalars, accumulated in FP64.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check
from .nufft import NufftPlan, _stream_ptr, _torch

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class SenseSystem:
    """A = Asense(G, sens) with R = Reg1(mask, 'beta', beta) (quadratic).

    G: NufftPlan with ncol = coils, one slice per problem (2D).
    sens: device complex64 [S, N2, N1, C]; beta: S values (or one).
    Images are [S, N2, N1] complex64, data [Mtot, C] complex64, on the device.
    """

    def __init__(self, G: NufftPlan, sens, beta, stream=None):
        torch = _torch()
        if G.D != 2:
            raise ValueError("CG-SENSE is provided for 2D plans")
        self.G, self.lib = G, G.lib
        self.S, self.C = G.nslice, G.ncol
        self.N1, self.N2 = int(G.Nd[0]), int(G.Nd[1])
        self.image_shape = (self.S, self.N2, self.N1)
        self.sens = sens.to(torch.complex64).contiguous()
        if tuple(self.sens.shape) != (self.S, self.N2, self.N1, self.C):
            raise ValueError("sens must be [S, N2, N1, C]")
        self.beta = np.ascontiguousarray(np.broadcast_to(np.asarray(beta, np.float64), (self.S,)))
        h = C.c_void_p()
        check(self.lib.mirt_sense_create(C.byref(h), G.handle, _ptr(self.sens),
                                         self.beta.ctypes.data_as(_dp), _stream_ptr(stream)))
        self.handle = h

    def forward(self, x, out=None, stream=None):
        torch = _torch()
        out = torch.empty((self.G.Mtot, self.C), dtype=torch.complex64, device="cuda") if out is None else out
        check(self.lib.mirt_sense_forward(self.handle, _ptr(x.contiguous()), _ptr(out), _stream_ptr(stream)))
        return out

    def adjoint(self, y, out=None, stream=None):
        torch = _torch()
        out = torch.empty(self.image_shape, dtype=torch.complex64, device="cuda") if out is None else out
        check(self.lib.mirt_sense_adjoint(self.handle, _ptr(y.contiguous()), _ptr(out), _stream_ptr(stream)))
        return out

    def reg(self, x, out=None, stream=None):
        torch = _torch()
        out = torch.empty(self.image_shape, dtype=torch.complex64, device="cuda") if out is None else out
        check(self.lib.mirt_sense_reg(self.handle, _ptr(x.contiguous()), _ptr(out), _stream_ptr(stream)))
        return out

    def toeplitz(self, stream=None):
        """Attach the Toeplitz Gram operator (Gnufft_gram) and the circulant
        preconditioner built from it; needed by pcg(precon=True / gram=True)."""
        check(self.lib.mirt_sense_toeplitz(self.handle, self.G.om_f.ctypes.data_as(_dp),
                                           _stream_ptr(stream)))
        self.has_toeplitz = True
        return self

    def precon_dcf(self, w, blend=1.0, stream=None):
        """Replace the circulant preconditioner by the one built from the
        density-compensation weights w (device FP64 [Mtot], e.g. the learned
        DCF), blended with the unweighted one (see mirt_sense_precon_dcf);
        blend=0 restores the unweighted preconditioner.  Needs toeplitz()."""
        check(self.lib.mirt_sense_precon_dcf(self.handle, self.G.om_f.ctypes.data_as(_dp),
                                             _ptr(w.to(_torch().float64).contiguous()),
                                             float(blend), _stream_ptr(stream)))
        return self

    def pcg(self, x, y, niter, W=None, precon=False, gram=False, xref=None, timing=False,
            stream=None):
        """niter iterations of qpwls_pcg1 (NUFFT pair each iteration) or, with
        gram=True, of qpwls_pcg2 on the Toeplitz normal equations; precon=True
        uses the circulant preconditioner.  In place on x; returns (nrmse, ms)
        as cg() does."""
        torch = _torch()
        Wf = None if W is None else W.to(torch.float32).contiguous()
        flags = (1 if precon else 0) | (2 if gram else 0)
        nr = np.zeros((niter + 1, self.S)) if xref is not None else None
        ms = np.zeros(max(niter, 1), dtype=np.float32) if timing else None
        check(self.lib.mirt_sense_pcg(self.handle, _ptr(x), _ptr(y.contiguous()), _ptr(Wf),
                                      int(niter), flags,
                                      _ptr(None if xref is None else xref.contiguous()),
                                      None if nr is None else nr.ctypes.data_as(_dp),
                                      None if ms is None else ms.ctypes.data_as(_fp),
                                      _stream_ptr(stream)))
        return nr, (ms[:niter] if timing else None)

    def warm_start(self, y, W=None, stream=None):
        """x0 = a A'(W y) per problem with the least-squares scale a."""
        torch = _torch()
        x = torch.empty(self.image_shape, dtype=torch.complex64, device="cuda")
        Wf = None if W is None else W.to(torch.float32).contiguous()
        check(self.lib.mirt_sense_warm_start(self.handle, _ptr(x), _ptr(y.contiguous()), _ptr(Wf),
                                             _stream_ptr(stream)))
        return x

    def cg(self, x, y, niter, W=None, xref=None, timing=False, stream=None):
        """niter qpwls_pcg1 iterations in place on x; returns (nrmse [niter+1, S]
        or None, device ms after each iteration or None)."""
        torch = _torch()
        Wf = None if W is None else W.to(torch.float32).contiguous()
        nr = np.zeros((niter + 1, self.S)) if xref is not None else None
        ms = np.zeros(max(niter, 1), dtype=np.float32) if timing else None
        check(self.lib.mirt_sense_cg(self.handle, _ptr(x), _ptr(y.contiguous()), _ptr(Wf),
                                     int(niter), _ptr(None if xref is None else xref.contiguous()),
                                     None if nr is None else nr.ctypes.data_as(_dp),
                                     None if ms is None else ms.ctypes.data_as(_fp),
                                     _stream_ptr(stream)))
        return nr, (ms[:niter] if timing else None)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mirt_sense_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Gram:
    """T = Gnufft_gram(G, W): the Toeplitz-embedded Gram operator G'WG of a 2D
    plan's trajectory (systems/Gnufft_gram.m), applied by two FFTs of the
    2N-padded image per column.  W: device FP64 [Mtot] weights or None;
    ncol: columns of the images it is applied to ([S, N2, N1, ncol])."""

    def __init__(self, G: NufftPlan, W=None, ncol=1, stream=None):
        self.lib = G.lib
        self.S, self.ncol = G.nslice, int(ncol)
        self.shape = (G.nslice, int(G.Nd[1]), int(G.Nd[0]), self.ncol)
        mo = G.slice_moff
        h = C.c_void_p()
        check(self.lib.mirt_toeplitz_create(
            C.byref(h), G.om_f.ctypes.data_as(_dp), G.Mtot,
            None if mo is None else mo.ctypes.data_as(C.POINTER(C.c_int64)), G.nslice,
            G.Nd.ctypes.data_as(C.POINTER(C.c_int32)), G.Kd.ctypes.data_as(C.POINTER(C.c_int32)),
            G.Jd.ctypes.data_as(C.POINTER(C.c_int32)), G.Ld.ctypes.data_as(C.POINTER(C.c_int32)),
            _ptr(None if W is None else W.contiguous()), self.ncol, _stream_ptr(stream)))
        self.handle = h

    def apply(self, x, out=None, stream=None):
        torch = _torch()
        out = torch.empty(self.shape, dtype=torch.complex64, device="cuda") if out is None else out
        check(self.lib.mirt_toeplitz_apply(self.handle, _ptr(x.contiguous()), _ptr(out),
                                           _stream_ptr(stream)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mirt_toeplitz_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def Gnufft_gram(G: NufftPlan, W=None, ncol=1):
    """[T, reuse] = Gnufft_gram(A, W) (systems/Gnufft_gram.m) for a table plan."""
    return Gram(G, W, ncol)


def Asense(G: NufftPlan, sens, beta=0.0):
    """A_mc = Asense(A, sens) (systems/Asense.m), with the Reg1 beta attached."""
    return SenseSystem(G, sens, beta)


def qpwls_pcg1(x, A: SenseSystem, W, yi, niter=1, xref=None):
    """[xs, info] = qpwls_pcg1(x, A, W, yi, C, 'niter', niter) with C the
    attached Reg1 penalty and precon = 1.  x (device) is updated in place and
    returned with the per-iteration NRMSE to xref (if given) as info."""
    nr, _ = A.cg(x, yi, niter, W=W, xref=xref)
    return x, nr


def trace_beta(M, sens, scale=2.0 ** -8):
    """beta_s = scale * trace(A_s'A_s) / np ~ scale * M_s * mean_n sum_c |s_c(n)|^2
    per problem s (the NUFFT Gram diagonal is M_s for M_s samples per coil)."""
    torch = _torch()
    p = (sens.abs() ** 2).sum(-1).to(torch.float64)
    return scale * np.asarray(M, np.float64) * p.reshape(p.shape[0], -1).mean(1).cpu().numpy()
