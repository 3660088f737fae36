"""Parity oracle for MIRT's table-based NUFFT interpolation.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg, as the checker; the product never imports it.

Two FP64 CPU implementations of the same kernels sit behind one numpy API:

* ``impl="port"``: this project's restatement, oracle/interp_table.c
  (liboracle.so);
* ``impl="ref"``: the reference's own kernels nufft/table/interp*_table1_*.c,
  compiled unmodified from the reference sources by oracle/Makefile into
  oracle/_ref/libmirt_ref.so and driven like the mex gateways
  (nufft/table/interp2_table_mex.c:87-121).

``nufft_ref`` restates the MATLAB glue (tables, scaling factors, nufft /
nufft_adj, exact DTFT).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_PORT = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libmirt_ref.so")
_libs: dict[str, C.CDLL] = {}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


# the reference checkout whose nufft/table sources _ref/ is compiled from
# (MIRT_REFERENCE overrides it); absent on hosts that only run the prebuilt _ref/
REF_TREE = os.environ.get("MIRT_REFERENCE", "/root/reference")


def build(quiet: bool = True) -> None:
    """Compile liboracle.so and, when the reference sources exist, _ref/libmirt_ref.so."""
    cmd = ["make", "-C", HERE]
    if os.path.isdir(os.path.join(REF_TREE, "nufft", "table")):
        cmd.append(f"REF={REF_TREE}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def ref_available() -> bool:
    return os.path.exists(_REF)


def _lib(impl: str) -> C.CDLL:
    if impl not in _libs:
        path = _PORT if impl == "port" else _REF
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        if impl == "port":
            for fn in (lib.oracle_interp_for, lib.oracle_interp_adj):
                fn.restype = C.c_int
        else:
            lib.ref_interp_cols.restype = C.c_int
            lib.ref_max_threads.restype = C.c_int
        _libs[impl] = lib
    return _libs[impl]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _tables(h):
    """split complex/real tables -> (keep-alive list, hr**, hi** or None)."""
    keep = []
    is_cx = any(np.iscomplexobj(t) for t in h)
    hr = (_dp * len(h))()
    hi = (_dp * len(h))() if is_cx else None
    for d, t in enumerate(h):
        r = np.ascontiguousarray(np.real(t), dtype=np.float64)
        keep.append(r)
        hr[d] = _dptr(r)
        if is_cx:
            i = np.ascontiguousarray(np.imag(t), dtype=np.float64)
            keep.append(i)
            hi[d] = _dptr(i)
    return keep, hr, hi


def _ints(v):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.int32).ravel(), dtype=np.intc)
    return a, a.ctypes.data_as(_ip)


def interp_for(ck, h, J, L, tm, K, order=0, impl="port", nthreads=1):
    """fm [M, N] = table interpolation of ck [prod(K), N] (column-major grid)."""
    ck = np.asarray(ck, dtype=np.complex128)
    if ck.ndim == 1:
        ck = ck[:, None]
    tm = np.asarray(tm, dtype=np.float64)
    tm = np.asfortranarray(tm.reshape(tm.shape[0], -1) if tm.ndim != 2 else tm)
    D = tm.shape[1]
    M, N = tm.shape[0], ck.shape[1]
    keep, hr, hi = _tables(h)
    Ka, Kp = _ints(K)
    Ja, Jp = _ints(J)
    La, Lp = _ints(L)
    rck = np.asfortranarray(ck.real)
    ick = np.asfortranarray(ck.imag)
    rfm = np.zeros((M, N), order="F")
    ifm = np.zeros((M, N), order="F")
    if impl == "port":
        lib = _lib("port")
        for n in range(N):
            rc = lib.oracle_interp_for(D, Kp, hr, hi, Jp, Lp, int(order), _dptr(tm), M,
                                       _dptr(rck[:, n]), _dptr(ick[:, n]),
                                       _dptr(rfm[:, n]), _dptr(ifm[:, n]))
            if rc:
                raise ValueError(f"oracle_interp_for failed ({rc})")
    else:
        rc = _lib("ref").ref_interp_cols(0, D, Kp, hr, hi, Jp, Lp, int(order), _dptr(tm), M, N,
                                         _dptr(rck), _dptr(ick), _dptr(rfm), _dptr(ifm),
                                         int(nthreads))
        if rc:
            raise ValueError("reference interp failed")
    del keep
    return rfm + 1j * ifm


def interp_adj(fm, h, J, L, tm, K, order=0, impl="port", nthreads=1):
    """ck [prod(K), N] = adjoint table interpolation of fm [M, N]."""
    fm = np.asarray(fm, dtype=np.complex128)
    if fm.ndim == 1:
        fm = fm[:, None]
    tm = np.asarray(tm, dtype=np.float64)
    tm = np.asfortranarray(tm.reshape(tm.shape[0], -1) if tm.ndim != 2 else tm)
    D = tm.shape[1]
    M, N = fm.shape
    nk = int(np.prod(K))
    keep, hr, hi = _tables(h)
    Ka, Kp = _ints(K)
    Ja, Jp = _ints(J)
    La, Lp = _ints(L)
    rfm = np.asfortranarray(fm.real)
    ifm = np.asfortranarray(fm.imag)
    rck = np.zeros((nk, N), order="F")
    ick = np.zeros((nk, N), order="F")
    if impl == "port":
        lib = _lib("port")
        for n in range(N):
            rc = lib.oracle_interp_adj(D, Kp, hr, hi, Jp, Lp, int(order), _dptr(tm), M,
                                       _dptr(rfm[:, n]), _dptr(ifm[:, n]),
                                       _dptr(rck[:, n]), _dptr(ick[:, n]))
            if rc:
                raise ValueError(f"oracle_interp_adj failed ({rc})")
    else:
        rc = _lib("ref").ref_interp_cols(1, D, Kp, hr, hi, Jp, Lp, int(order), _dptr(tm), M, N,
                                         _dptr(rck), _dptr(ick), _dptr(rfm), _dptr(ifm),
                                         int(nthreads))
        if rc:
            raise ValueError("reference interp_adj failed")
    del keep
    return rck + 1j * ick


def ref_max_threads() -> int:
    return int(_lib("ref").ref_max_threads())
