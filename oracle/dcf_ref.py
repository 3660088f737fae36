"""FP64 restatement of MIRT's density compensation (mri/ir_mri_density_comp.m).

TEST INFRASTRUCTURE ONLY (the checker of mirt_dcf_pipe / mirt_dcf_jackson).

The interpolator P is the reference's table pair: ``oracle.interp_adj`` and
``oracle.interp_for`` (the reference's own C kernels from oracle/_ref when they
were built, else the bit-identical restatement), wrapped with the phase shift
as nufft/nufft_table_interp.m:75-78 and nufft/nufft_table_adj.m:47-50 do.
"""
from __future__ import annotations

import numpy as np

import oracle
from oracle import nufft_ref as nr


def _impl():
    return "ref" if oracle.ref_available() else "port"


def ppt(w, st, nthreads=8):
    """P P' w for a table NUFFT structure ``st`` (nufft_ref.nufft_init_table)."""
    X = np.asarray(w, dtype=np.complex128)
    ph = st["phase_shift"]
    if ph is not None:
        X = X * np.conj(ph)
    ck = oracle.interp_adj(X[:, None], st["h"], st["Jd"], st["Ld"], st["tm"], st["Kd"], 0,
                           impl=_impl(), nthreads=nthreads)
    g = oracle.interp_for(ck, st["h"], st["Jd"], st["Ld"], st["tm"], st["Kd"], 0,
                          impl=_impl(), nthreads=nthreads)[:, 0]
    if ph is not None:
        g = g * ph
    return g


def _interp_adj_fn(X, st):
    return oracle.interp_adj(np.asarray(X)[:, None], st["h"], st["Jd"], st["Ld"], st["tm"],
                             st["Kd"], 0, impl=_impl(), nthreads=8)[:, 0]


def dcf_pipe(st, niter=20, thresh=0.02, fov=1.0, wi=None):
    """ir_mri_dcf_pipe_do (mri/ir_mri_density_comp.m:203-281) with unitv = [] and
    isave = []: returns (wi, iterations, last max |goal - 1|)."""
    M = st["M"]
    d = len(st["Nd"])
    fov = np.broadcast_to(np.asarray(fov, dtype=np.float64), (d,))
    w = np.ones(M) if wi is None else np.asarray(wi, dtype=np.float64).copy()
    goal = np.inf
    it = 0
    resid = np.inf
    # while (max(abs(goal-1)) > thresh)  (:231)
    while resid > thresh:
        it += 1
        goal = np.real(ppt(w, st))                     # (:233-240)
        if np.any(goal <= 0):
            raise RuntimeError("pipe bug")             # (:241-243)
        w = w / goal                                   # (:244)
        resid = np.max(np.abs(goal - 1)) if M else 0.0
        if it > niter:                                 # (:245-248)
            break
    # scale: sum(psf) = prod(N ./ fov)  (:258-261)
    psf = nr.nufft_adj(w, st, _interp_adj_fn)
    scale = np.prod(np.asarray(st["Nd"]) / fov) / np.sum(np.real(psf))
    return scale * w, it, resid


def dcf_jackson(st):
    """wi = 1 ./ real(P (P' 1)) (mri/ir_mri_density_comp.m:171-174)."""
    return 1.0 / np.real(ppt(np.ones(st["M"]), st))
