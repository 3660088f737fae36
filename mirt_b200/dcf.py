"""Density compensation on the device NUFFT: ir_mri_density_comp('pipe' | 'jackson').

Mirrors mri/ir_mri_density_comp.m: ``wi = ir_mri_density_comp(kspace, dtype,
G=..., arg_pipe={...})``.  ``G`` is a single-column :class:`NufftPlan` (the
reference's Gnufft object, whose ``st`` carries the table interpolator); its
slices are independent trajectories and each gets its own weights.  The
Voronoi method is geometry on the host (voronoin / convhulln) and is not
provided here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check
from .nufft import NufftPlan, _stream_ptr, _torch

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)


def dcf_pipe(G: NufftPlan, niter=20, thresh=0.02, fov=1.0, wi=None, stream=None,
             return_info=False):
    """Pipe & Menon weights (ir_mri_dcf_pipe_do, mri/ir_mri_density_comp.m:203-281).

    Returns a device FP64 tensor [Mtot] (and, with ``return_info``, the updates
    done and the last max |goal - 1| per slice).  ``wi`` (device FP64 [Mtot])
    replaces the initial w = 1, like the reference's 'wi' option.
    """
    torch = _torch()
    if G.ncol != 1:
        raise ValueError("density compensation needs a single-column NUFFT plan (ncol = 1)")
    fov = np.ascontiguousarray(np.broadcast_to(np.asarray(fov, dtype=np.float64), (G.D,)))
    if wi is None:
        w = torch.empty(G.Mtot, dtype=torch.float64, device="cuda")
        init = 1
    else:
        w = wi.detach().to(device="cuda", dtype=torch.float64).contiguous().clone()
        if w.numel() != G.Mtot:
            raise ValueError("wi must have one entry per sample")
        init = 0
    iters = np.zeros(G.nslice, dtype=np.int32)
    resid = np.zeros(G.nslice, dtype=np.float64)
    check(G.lib.mirt_dcf_pipe(G.handle, C.c_void_p(w.data_ptr()), init, int(niter), float(thresh),
                              fov.ctypes.data_as(_dp), iters.ctypes.data_as(_i32p),
                              resid.ctypes.data_as(_dp), _stream_ptr(stream)))
    if return_info:
        return w, iters, resid
    return w


def dcf_jackson(G: NufftPlan, stream=None):
    """w = 1 ./ real(P (P' 1)) (ir_mri_dcf_jackson, mri/ir_mri_density_comp.m:160-180)."""
    torch = _torch()
    if G.ncol != 1:
        raise ValueError("density compensation needs a single-column NUFFT plan (ncol = 1)")
    w = torch.empty(G.Mtot, dtype=torch.float64, device="cuda")
    check(G.lib.mirt_dcf_jackson(G.handle, C.c_void_p(w.data_ptr()), _stream_ptr(stream)))
    return w


def ir_mri_density_comp(kspace, dtype, G: NufftPlan | None = None, arg_pipe=None, fix_edge=2):
    """wi = ir_mri_density_comp(kspace, dtype, 'G', G, 'arg_pipe', {...}) as numpy FP64 [M].

    ``kspace`` [M, d] fixes M and d, as in the reference (the sample locations
    themselves live in G).  ``arg_pipe``: dict with the reference's options
    niter (20), thresh (0.02), fov (1), wi (None).
    """
    kspace = np.asarray(kspace)
    if dtype == "voronoi":
        raise NotImplementedError("voronoi weights (host geometry) are not provided")
    if dtype not in ("pipe", "jackson"):
        raise ValueError(f"unknown DCF type {dtype}")
    if G is None:
        raise ValueError(f"'{dtype}' needs the NUFFT object G")
    if kspace.ndim != 2 or kspace.shape[0] != G.Mtot or kspace.shape[1] != G.D:
        raise ValueError("kspace must be [M, d] for the M samples of G")
    if dtype == "jackson":
        return dcf_jackson(G).cpu().numpy()
    a = dict(niter=20, thresh=0.02, fov=1.0, wi=None)
    a.update(arg_pipe or {})
    fov = np.asarray(a["fov"], dtype=np.float64).ravel()
    if fov.size not in (1, G.D):
        raise ValueError("bad fov")
    wi = a["wi"]
    if wi is not None:
        torch = _torch()
        wi = torch.as_tensor(np.asarray(wi, dtype=np.float64)).cuda()
    return dcf_pipe(G, a["niter"], a["thresh"], fov, wi).cpu().numpy()
