"""Python mirror of the eight mex gateways of nufft/table/.

Same names, argument order and meaning as the MATLAB calls

    fm = interp2_table_mex(ck, h1, h2, J, L, tm, [order, flips])
    ck = interp2_table_adj_mex(fm, h1, h2, J, L, tm, K, [order, flips])

with numpy arrays in the roles of the mxArrays: complex128 for complex
double, float64 for real double, int32 for the integer arguments.  Argument
errors raise :class:`MexError` with the gateway's mexFail() text followed by
the Fail() diagnostic, e.g. ``interp2_table_mex failed: h1 size problem``.
Outputs have the gateway's shape: fm [M, N], ck [prod(K), N].

Every call runs on the GPU through libmirt_b200.so (FP32 arithmetic with
FP64 table-index selection); there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import MIRT_ERR_ARG, MirtError, check, load

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


class MexError(MirtError):
    """A gateway argument error (the reference's mexErrMsgTxt)."""


def _p(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def _is_complex_double(a) -> bool:
    return isinstance(a, np.ndarray) and a.dtype == np.complex128


def _is_real_double(a) -> bool:
    return isinstance(a, np.ndarray) and a.dtype == np.float64


def _split(a):
    """column-major real / imag FP64 copies (mxGetPr / mxGetPi)."""
    f = a.ravel(order="F")
    return np.ascontiguousarray(f.real), np.ascontiguousarray(f.imag)


def _int32(a, name, n, msg, fail):
    if not (isinstance(a, np.ndarray) and a.dtype == np.int32 and a.size == n):
        raise MexError(MIRT_ERR_ARG, f"{fail}: {msg}")
    return np.ascontiguousarray(a.ravel(), dtype=np.int32)


def _opt_int32(a, n, msg, fail):
    if a is None:
        return None, 0
    return _int32(a, "", n, msg, fail), n


def _table(h):
    """(re, im|None, rows, cols) of a real or complex double table."""
    if not isinstance(h, np.ndarray) or h.dtype not in (np.float64, np.complex128):
        return None
    rows = h.shape[0] if h.ndim >= 1 else 1
    cols = int(np.prod(h.shape[1:])) if h.ndim > 1 else 1
    if h.dtype == np.complex128:
        re, im = _split(h)
        return re, im, rows, cols
    return np.ascontiguousarray(h.ravel(order="F")), None, rows, cols


def _tables(hs, fail):
    out = []
    for h in hs:
        t = _table(h)
        if t is None:
            raise MexError(MIRT_ERR_ARG, f"{fail}: h must be real or complex double (preferably real)")
        out.append(t)
    return out


def _call(fn, *args):
    rc = fn(*args)
    if rc == MIRT_ERR_ARG:
        msg = load().mirt_last_error().decode(errors="replace")
        raise MexError(rc, msg)
    check(rc)


def _fwd(D, ck, hs, J, L, tm, order, flips, fail, jmsg, lmsg, fmsg):
    if not _is_complex_double(ck):
        raise MexError(MIRT_ERR_ARG, f"{fail}: mxIsComplexDouble")
    if not _is_real_double(tm):
        raise MexError(MIRT_ERR_ARG, f"{fail}: mxIsRealDouble")
    Jd = _int32(J, "J", D, jmsg, fail)
    Ld = _int32(L, "L", D, lmsg, fail)
    od, on = _opt_int32(order, 1, "order must be scalar int32 (0 | 1)", fail)
    fd, fn_ = _opt_int32(flips, D, fmsg, fail)
    tabs = _tables(hs, fail)
    tm2 = tm.reshape(tm.shape[0], -1) if tm.ndim != 2 else tm
    tmf = np.ascontiguousarray(tm2.ravel(order="F"))
    M, tcols = tm2.shape
    re, im = _split(ck)
    lib = load()
    if D == 1:
        K1 = ck.shape[0]
        N = int(np.prod(ck.shape[1:])) if ck.ndim > 1 else 1
        N_out = N
    else:
        dims = np.array(ck.shape if ck.ndim else (1,), dtype=np.int64)
        N_out = int(dims[D]) if len(dims) > D else 1
    fm_re = np.zeros(M * N_out)
    fm_im = np.zeros(M * N_out)
    targs = []
    for r, i, rows, cols in tabs:
        targs += [_p(r), _p(i), rows, cols]
    common = [_p(Jd, _i32p), D, _p(Ld, _i32p), D, _p(tmf), M, tcols,
              _p(od, _i32p), on, _p(fd, _i32p), fn_, _p(fm_re), _p(fm_im)]
    if D == 1:
        _call(lib.mirt_interp1_table_mex, _p(re), _p(im), K1, N, *targs, *common)
    else:
        fn = {2: lib.mirt_interp2_table_mex, 3: lib.mirt_interp3_table_mex,
              4: lib.mirt_interp4_table_mex}[D]
        _call(fn, _p(re), _p(im), _p(dims, _i64p), len(dims), *targs, *common)
    return (fm_re + 1j * fm_im).reshape((M, N_out), order="F")


def _adj(D, fm, hs, J, L, tm, K, order, flips, fail, jmsg, lmsg, kmsg, fmsg):
    if not _is_complex_double(fm):
        raise MexError(MIRT_ERR_ARG, f"{fail}: mxIsComplexDouble")
    if not _is_real_double(tm):
        raise MexError(MIRT_ERR_ARG, f"{fail}: mxIsRealDouble")
    Jd = _int32(J, "J", D, jmsg, fail)
    Kd = _int32(K, "K", D, kmsg, fail)
    Ld = _int32(L, "L", D, lmsg, fail)
    od, on = _opt_int32(order, 1, "order must be scalar int32 (0 | 1)", fail)
    fd, fn_ = _opt_int32(flips, D, fmsg, fail)
    tabs = _tables(hs, fail)
    tm2 = tm.reshape(tm.shape[0], -1) if tm.ndim != 2 else tm
    tmf = np.ascontiguousarray(tm2.ravel(order="F"))
    fm2 = fm.reshape(fm.shape[0], -1) if fm.ndim != 2 else fm
    M, N = fm2.shape
    re, im = _split(fm2)
    nk = int(np.prod(Kd.astype(np.int64)))
    ck_re = np.zeros(nk * N)
    ck_im = np.zeros(nk * N)
    targs = []
    for r, i, rows, cols in tabs:
        targs += [_p(r), _p(i), rows, cols]
    lib = load()
    fn = {1: lib.mirt_interp1_table_adj_mex, 2: lib.mirt_interp2_table_adj_mex,
          3: lib.mirt_interp3_table_adj_mex, 4: lib.mirt_interp4_table_adj_mex}[D]
    _call(fn, _p(re), _p(im), M, N, *targs, _p(Jd, _i32p), D, _p(Ld, _i32p), D,
          _p(tmf), tm2.shape[0], tm2.shape[1], _p(Kd, _i32p), D,
          _p(od, _i32p), on, _p(fd, _i32p), fn_, _p(ck_re), _p(ck_im))
    return (ck_re + 1j * ck_im).reshape((nk, N), order="F")


def interp1_table_mex(ck, h, J, L, tm, order=None, flips=None):
    """fm = interp1_table_mex(ck, h, J, L, tm, [order, flips]); nufft/table/interp1_table_mex.c."""
    return _fwd(1, ck, [h], J, L, tm, order, flips, "interp1_table_mex() failed",
                "J must be scalar int32", "L must be scalar int32",
                "flips must be scalar int32 (0 | 1)")


def interp2_table_mex(ck, h1, h2, J, L, tm, order=None, flips=None):
    """fm = interp2_table_mex(ck, h1, h2, J, L, tm, [order, flips]); nufft/table/interp2_table_mex.c."""
    return _fwd(2, ck, [h1, h2], J, L, tm, order, flips, "interp2_table_mex failed",
                "J must be [1,2]", "L must be [1,2]", "flips must be [1 2] int32 (0 | 1)")


def interp3_table_mex(ck, h1, h2, h3, J, L, tm, order=None, flips=None):
    """fm = interp3_table_mex(ck, h1, h2, h3, J, L, tm, [order, flips]); nufft/table/interp3_table_mex.c."""
    return _fwd(3, ck, [h1, h2, h3], J, L, tm, order, flips, "interp3_table_mex failed",
                "J must be [1,3]", "L must be [1,3]", "flips must be [1 3] int32 (0 | 1)")


def interp4_table_mex(ck, h1, h2, h3, h4, J, L, tm, order=None, flips=None):
    """fm = interp4_table_mex(ck, h1, h2, h3, h4, J, L, tm, [order, flips]);
    nufft/table/interp4_table_mex.c (whose failure text names interp3_table_mex)."""
    return _fwd(4, ck, [h1, h2, h3, h4], J, L, tm, order, flips, "interp3_table_mex failed",
                "J must be [1,4]", "L must be [1,4]", "flips must be [1 4] int32 (0 | 1)")


def interp1_table_adj_mex(fm, h, J, L, tm, K, order=None, flips=None):
    """ck = interp1_table_adj_mex(fm, h, J, L, tm, K, [order, flips])."""
    return _adj(1, fm, [h], J, L, tm, K, order, flips, "interp1_table_adj_mex() failed",
                "J must be scalar int32", "L must be scalar int32", "K must be scalar int32",
                "flips must be scalar int32 (0 | 1)")


def interp2_table_adj_mex(fm, h1, h2, J, L, tm, K, order=None, flips=None):
    """ck = interp2_table_adj_mex(fm, h1, h2, J, L, tm, K, [order, flips])."""
    return _adj(2, fm, [h1, h2], J, L, tm, K, order, flips, "interp2_table_adj_mex() failed",
                "J must be int32 [1,2]", "L must be int32 [1,2]", "K must be int32 [1,2]",
                "flips must be [1 2] int32 (0 | 1)")


def interp3_table_adj_mex(fm, h1, h2, h3, J, L, tm, K, order=None, flips=None):
    """ck = interp3_table_adj_mex(fm, h1, h2, h3, J, L, tm, K, [order, flips])."""
    return _adj(3, fm, [h1, h2, h3], J, L, tm, K, order, flips, "interp3_table_adj_mex() failed",
                "J must be int32 [1,3]", "L must be int32 [1,3]", "K must be int32 [1,3]",
                "flips must be [1 3] int32 (0 | 1)")


def interp4_table_adj_mex(fm, h1, h2, h3, h4, J, L, tm, K, order=None, flips=None):
    """ck = interp4_table_adj_mex(fm, h1, h2, h3, h4, J, L, tm, K, [order, flips])."""
    return _adj(4, fm, [h1, h2, h3, h4], J, L, tm, K, order, flips,
                "interp4_table_adj_mex() failed", "J must be int32 [1,4]", "L must be int32 [1,4]",
                "K must be int32 [1,4]", "flips must be [1 4] int32 (0 | 1)")
