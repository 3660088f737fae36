"""Device-resident interpolation plans and the table NUFFT, over torch tensors.

The MATLAB-style entry points mirror the reference's NUFFT interface:

    st = nufft_init(om, Nd, Jd, Kd, n_shift, 'table', Ld, 'minmax:kb')
    X  = nufft(x, st)        # nufft/nufft.m:128-165
    x  = nufft_adj(X, st)    # nufft/nufft_adj.m:32-80

with numpy inputs and outputs in MATLAB index order (x[n1, n2, (n3), coil]).
``NufftPlan`` and ``InterpPlan`` are the device-resident forms used by the
solvers and the benchmark: complex64 torch tensors on the GPU with the coil
index innermost.  torch provides device memory and streams only; all compute
runs in libmirt_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def _torch():
    import torch
    return torch


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _i32(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32).ravel())


def _moff(slice_moff, Mtot):
    if slice_moff is None:
        return None, 1
    mo = np.ascontiguousarray(np.asarray(slice_moff, dtype=np.int64))
    if mo[0] != 0 or mo[-1] != Mtot:
        raise ValueError("slice offsets must start at 0 and end at Mtot")
    return mo, len(mo) - 1


def minmax_kb_table(N: int, J: int, K: int, L: int) -> np.ndarray:
    """Complex min-max:KB table st.h{d} (length J*L+1) built by the library in FP64."""
    n = J * L + 1
    re, im = np.zeros(n), np.zeros(n)
    check(load().mirt_minmax_kb_table(N, J, K, L, re.ctypes.data_as(_dp), im.ctypes.data_as(_dp)))
    return re + 1j * im


def minmax_kb_scale(N: int, J: int, K: int) -> np.ndarray:
    """1D scaling factors nufft_scale(N, K, alpha, beta) with the min-max:KB fit."""
    re, im = np.zeros(N), np.zeros(N)
    check(load().mirt_minmax_kb_scale(N, J, K, re.ctypes.data_as(_dp), im.ctypes.data_as(_dp)))
    return re + 1j * im


def _plan_config(lib, handle) -> dict:
    v = (C.c_int32 * 23)()
    check(lib.mirt_interp_plan_config(handle, v, 23))
    return {"spread_tile": [v[0], v[1], v[2]], "spread_threads": v[3], "spread_heavy_first": v[4],
            "coil_lanes": v[5], "gather_threads": v[6],
            "gather_ctas": v[8], "sort_bin": [v[9], v[10], v[11]], "split_chunk": v[12],
            "spread_tasks": v[13], "spread_padc": v[14], "spread_reductions": v[15],
            "spread_atomic": v[16], "spread_own": v[17], "spread_sweep": v[18],
            "spread_sweep_rows": v[19], "gather_tma": v[20], "spread_dense": v[21],
            "spread_staged": v[22]}


class InterpPlan:
    """Plan of the table gather / spread for fixed tables and trajectory.

    tm: [Mtot, D] float64 (t = omega / (2 pi / K)), D = 1..4; tables: list of
    D arrays (complex128 or float64).  Device tensors: grid [nslice, K_D, ...,
    K_1, ncol] and samples [Mtot, ncol], complex64, contiguous.  A 4D plan
    runs on a 3D plan of the grids' hyperplanes; its setters tune that plan.
    """

    def __init__(self, K, J, L, tables, tm, ncol, order=0, slice_moff=None, phase=None,
                 stream=None):
        torch = _torch()
        self.lib = load()
        tm = np.asarray(tm, dtype=np.float64)
        if tm.ndim == 1:
            tm = tm[:, None]
        self.D = tm.shape[1]
        self.K, self.J, self.L = _i32(K), _i32(J), _i32(L)
        self.Mtot = tm.shape[0]
        self.ncol = int(ncol)
        mo, self.nslice = _moff(slice_moff, self.Mtot)
        is_cx = any(np.iscomplexobj(h) for h in tables)
        self._keep = []
        hr = (_dp * max(3, self.D))()
        hi = (_dp * max(3, self.D))() if is_cx else None
        for d, h in enumerate(tables):
            r = np.ascontiguousarray(np.real(h), dtype=np.float64)
            self._keep.append(r)
            hr[d] = r.ctypes.data_as(_dp)
            if is_cx:
                i = np.ascontiguousarray(np.imag(h), dtype=np.float64)
                self._keep.append(i)
                hi[d] = i.ctypes.data_as(_dp)
        tmf = np.ascontiguousarray(tm.ravel(order="F"))
        pr = pi = None
        if phase is not None:
            phase = np.asarray(phase, dtype=np.complex128)
            pr = np.ascontiguousarray(phase.real)
            pi = np.ascontiguousarray(phase.imag)
        h = C.c_void_p()
        check(self.lib.mirt_interp_plan_create(
            C.byref(h), self.D, self.K.ctypes.data_as(_i32p), self.J.ctypes.data_as(_i32p),
            self.L.ctypes.data_as(_i32p), hr, hi, int(order), tmf.ctypes.data_as(_dp),
            self.Mtot, None if mo is None else mo.ctypes.data_as(_i64p), self.nslice,
            self.ncol, None if pr is None else pr.ctypes.data_as(_dp),
            None if pi is None else pi.ctypes.data_as(_dp), _stream_ptr(stream)))
        self.handle = h
        self._keep = []
        self.grid_shape = (self.nslice,) + tuple(int(k) for k in self.K[::-1]) + (self.ncol,)
        self.sample_shape = (self.Mtot, self.ncol)
        self.device = torch.device("cuda", torch.cuda.current_device())

    def forward(self, ck, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.sample_shape, dtype=torch.complex64, device=ck.device)
        assert ck.is_contiguous() and ck.dtype == torch.complex64
        check(self.lib.mirt_interp_plan_forward(self.handle, C.c_void_p(ck.data_ptr()),
                                                C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def adjoint(self, fm, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.grid_shape, dtype=torch.complex64, device=fm.device)
        assert fm.is_contiguous() and fm.dtype == torch.complex64
        check(self.lib.mirt_interp_plan_adjoint(self.handle, C.c_void_p(fm.data_ptr()),
                                                C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def autotune(self, stream=None):
        """Pick the fastest gather / spread launch shapes for this trajectory."""
        check(self.lib.mirt_interp_plan_autotune(self.handle, _stream_ptr(stream)))
        return self.config()

    def config(self):
        return _plan_config(self.lib, self.handle)

    def set_deterministic(self, deterministic=True):
        """False: the spread may add with shared-memory atomics (faster, not
        bitwise reproducible); the autotuner then also tries that variant."""
        check(self.lib.mirt_interp_plan_set_deterministic(self.handle, int(bool(deterministic))))
        return self.config()

    def set_ownership(self, own=True, stream=None):
        """Ownership spread (2D, J = 6; see mirt_interp_plan_set_ownership)."""
        check(self.lib.mirt_interp_plan_set_ownership(self.handle, int(bool(own)),
                                                      _stream_ptr(stream)))
        return self.config()

    def set_sweep(self, segments=1, rows=4):
        """Row-sweep spread (2D, J = 6; see mirt_interp_plan_set_sweep):
        uniform segments per grid row (True = 1; 0 / False = tiled spread;
        -1 = balanced team list) and grid rows per band (1, 2 or 4).  3D
        plans (J = 6, coil chunks of 8, 16 or 32): the line sweep with
        `segments` uniform segments per line block (rows unused)."""
        check(self.lib.mirt_interp_plan_set_sweep(self.handle, int(segments), int(rows)))
        return self.config()

    def set_gather(self, tma=True):
        """TMA-staged gather (2D, J = 6, even C >= 32) or the plain gather
        (see mirt_interp_plan_set_gather): True / 1 tiles of 32 coils, 2 tiles
        of 16 coils, False / 0 the plain gather."""
        check(self.lib.mirt_interp_plan_set_gather(self.handle, int(tma)))
        return self.config()

    def fault(self):
        """1 if an in-kernel wait ran out since the last call (see
        mirt_interp_plan_fault), else 0."""
        f = C.c_int32(0)
        check(self.lib.mirt_interp_plan_fault(self.handle, C.byref(f)))
        return f.value

    def set_dense(self, on=True):
        """Dense-bin patches in the 2D row sweep (see mirt_interp_plan_set_dense)."""
        check(self.lib.mirt_interp_plan_set_dense(self.handle, int(bool(on))))

    def set_staged(self, mode=1):
        """2D row sweep staged per bin column: 0 off, 1 after the ordering
        pass, 2 reading the caller's samples (see mirt_interp_plan_set_staged)."""
        check(self.lib.mirt_interp_plan_set_staged(self.handle, int(mode)))

    def set_fault_test(self, on=True):
        """Test hook of the TMA gather's bounded waits (see
        mirt_interp_plan_set_fault_test): no copies, every wait runs out."""
        check(self.lib.mirt_interp_plan_set_fault_test(self.handle, int(bool(on))))

    def set_spread(self, tile, threads=32, padc=0, stream=None):
        """Fix the spread tiling (tile extents per dimension, CTA size, spare
        tile columns 0 or J1 - 1) instead of autotuning it."""
        T = _i32(list(tile) + [1] * (3 - len(tile)))
        check(self.lib.mirt_interp_plan_set_spread(
            self.handle, T.ctypes.data_as(C.POINTER(C.c_int32)), int(threads), int(padc),
            _stream_ptr(stream)))
        return self.config()

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mirt_interp_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NufftPlan:
    """Table NUFFT with min-max:KB tables built in FP64 by the library.

    om: [Mtot, D] radians; Nd, Jd, Kd, Ld per dimension; n_shift (default 0).
    Device tensors: image [nslice, N_D, ..., N_1, ncol], samples [Mtot, ncol].
    """

    def __init__(self, om, Nd, Jd, Kd, n_shift=None, Ld=1024, ncol=1, slice_moff=None,
                 stream=None):
        torch = _torch()
        self.lib = load()
        om = np.asarray(om, dtype=np.float64)
        if om.ndim == 1:
            om = om[:, None]
        self.D = om.shape[1]
        D = self.D
        self.Nd, self.Jd, self.Kd = _i32(Nd), _i32(Jd), _i32(Kd)
        self.Ld = _i32(Ld if np.ndim(Ld) else [Ld] * D)
        self.n_shift = np.ascontiguousarray(
            np.zeros(D) if n_shift is None else np.asarray(n_shift, dtype=np.float64).ravel())
        self.Mtot = om.shape[0]
        self.ncol = int(ncol)
        mo, self.nslice = _moff(slice_moff, self.Mtot)
        omf = np.ascontiguousarray(om.ravel(order="F"))
        self.handle = self._create(omf, mo, stream)
        self.om_f = omf                      # trajectory, column-major FP64 (Toeplitz set-up)
        self.slice_moff = mo
        self.image_shape = (self.nslice,) + tuple(int(n) for n in self.Nd[::-1]) + (self.ncol,)
        self.sample_shape = (self.Mtot, self.ncol)

    def _create(self, omf, mo, stream):
        h = C.c_void_p()
        check(self.lib.mirt_nufft_create(
            C.byref(h), self.D, self.Nd.ctypes.data_as(_i32p), self.Kd.ctypes.data_as(_i32p),
            self.Jd.ctypes.data_as(_i32p), self.Ld.ctypes.data_as(_i32p),
            self.n_shift.ctypes.data_as(_dp), omf.ctypes.data_as(_dp), self.Mtot,
            None if mo is None else mo.ctypes.data_as(_i64p), self.nslice, self.ncol,
            _stream_ptr(stream)))
        return h

    def forward(self, x, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.sample_shape, dtype=torch.complex64, device=x.device)
        assert x.is_contiguous() and x.dtype == torch.complex64
        check(self.lib.mirt_nufft_forward(self.handle, C.c_void_p(x.data_ptr()),
                                          C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def adjoint(self, X, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.image_shape, dtype=torch.complex64, device=X.device)
        assert X.is_contiguous() and X.dtype == torch.complex64
        check(self.lib.mirt_nufft_adjoint(self.handle, C.c_void_p(X.data_ptr()),
                                          C.c_void_p(out.data_ptr()), _stream_ptr(stream)))
        return out

    def autotune(self, stream=None):
        """Pick the fastest gather / spread launch shapes for this trajectory."""
        check(self.lib.mirt_nufft_autotune(self.handle, _stream_ptr(stream)))
        return self.config()

    def set_deterministic(self, deterministic=True):
        """See InterpPlan.set_deterministic."""
        check(self.lib.mirt_interp_plan_set_deterministic(
            self.lib.mirt_nufft_interp_plan(self.handle), int(bool(deterministic))))
        return self.config()

    def set_sweep(self, segments=1, rows=4):
        """See InterpPlan.set_sweep."""
        check(self.lib.mirt_interp_plan_set_sweep(
            self.lib.mirt_nufft_interp_plan(self.handle), int(segments), int(rows)))
        return self.config()

    def set_dense(self, on=True):
        """See InterpPlan.set_dense."""
        check(self.lib.mirt_interp_plan_set_dense(self.lib.mirt_nufft_interp_plan(self.handle),
                                                  int(bool(on))))

    def set_staged(self, mode=1):
        """See InterpPlan.set_staged."""
        check(self.lib.mirt_interp_plan_set_staged(self.lib.mirt_nufft_interp_plan(self.handle),
                                                   int(mode)))

    def set_gather(self, tma=True):
        """See InterpPlan.set_gather."""
        check(self.lib.mirt_interp_plan_set_gather(self.lib.mirt_nufft_interp_plan(self.handle),
                                                   int(tma)))
        return self.config()

    def fault(self):
        """See InterpPlan.fault."""
        f = C.c_int32(0)
        check(self.lib.mirt_interp_plan_fault(self.lib.mirt_nufft_interp_plan(self.handle),
                                              C.byref(f)))
        return f.value

    def capture(self, x=None, X=None, xa=None):
        """CUDA graph of forward x -> X (if x) then adjoint X -> xa (if xa) on
        these buffers; replay with .launch(stream)."""
        return NufftGraph(self, x, X, xa)

    def config(self):
        return _plan_config(self.lib, self.lib.mirt_nufft_interp_plan(self.handle))

    def fft_config(self):
        """{'fused_fft': 1 if the FFT runs as the library's fused passes,
        'launches_forward', 'launches_adjoint': library kernels per call}."""
        v = (C.c_int32 * 3)()
        check(self.lib.mirt_nufft_config(self.handle, v, 3))
        return {"fused_fft": v[0], "launches_forward": v[1], "launches_adjoint": v[2]}

    def forward_host(self, x: np.ndarray, out: np.ndarray | None = None, stream=None):
        """host complex64 image (device layout) -> host complex64 samples."""
        x = np.ascontiguousarray(x, dtype=np.complex64)
        if out is None:
            out = np.empty(self.sample_shape, dtype=np.complex64)
        check(self.lib.mirt_nufft_forward_host(self.handle, x.ctypes.data_as(_fp),
                                               out.ctypes.data_as(_fp), _stream_ptr(stream)))
        return out

    def adjoint_host(self, X: np.ndarray, out: np.ndarray | None = None, stream=None):
        X = np.ascontiguousarray(X, dtype=np.complex64)
        if out is None:
            out = np.empty(self.image_shape, dtype=np.complex64)
        check(self.lib.mirt_nufft_adjoint_host(self.handle, X.ctypes.data_as(_fp),
                                               out.ctypes.data_as(_fp), _stream_ptr(stream)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mirt_nufft_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def newfft_kb_table(J: int, L: int) -> np.ndarray:
    """Real table of newfft's default 'kb:minmax' interpolator, [J*L+1]."""
    h = np.empty(int(J) * int(L) + 1)
    check(load().mirt_newfft_kb_table(int(J), int(L), h.ctypes.data_as(_dp)))
    return h


def newfft_kb_scale(N: int, J: int, K: int, nmid: float) -> np.ndarray:
    """1D scaling factors of newfft's 'kb:minmax' interpolator, [N]."""
    s = np.empty(int(N))
    check(load().mirt_newfft_kb_scale(int(N), int(J), int(K), float(nmid),
                                      s.ctypes.data_as(_dp)))
    return s


_KTYPES = {"kb:minmax": 0, "kb:beatty": 1, "diric": 2, "minmax:kb": 3, "minmax:unif": 4,
           "minmax:tuned": 5, "linear": 6}


_USER_KTYPES = ("kb:user", "minmax:user")


def _user_args(ktype, kb_alf, kb_m, alpha, beta):
    if ktype == "kb:user":
        if kb_alf is None or kb_m is None:
            raise ValueError("kb_alf and kb_m required")
        if float(kb_m) != int(kb_m):
            raise ValueError("kb:user: kb_m must be an integer")
        return float(kb_alf), int(kb_m)
    if alpha is None or beta is None:
        raise ValueError("user must provide alpha/beta")
    a = np.ascontiguousarray(np.atleast_1d(np.asarray(alpha, dtype=np.float64)))
    return a, float(beta)


def _newfft_table_complex(ktype, N, J, K, L, kb_alf, kb_m, alpha, beta):
    code = {**_KTYPES, "kb:user": 7, "minmax:user": 8}.get(ktype)
    if code is None:
        raise ValueError(f"ktype must be one of {sorted(_KTYPES) + list(_USER_KTYPES)}")
    a, m, al, b = 0.0, 0, None, 0.0
    if ktype == "kb:user":
        a, m = _user_args(ktype, kb_alf, kb_m, alpha, beta)
    elif ktype == "minmax:user":
        al, b = _user_args(ktype, kb_alf, kb_m, alpha, beta)
    hr = np.empty(int(J) * int(L) + 1)
    hi = np.empty_like(hr)
    check(load().mirt_newfft_table_complex(
        code, int(N), int(J), int(K), int(L), a, m,
        None if al is None else al.ctypes.data_as(_dp), 0 if al is None else al.size, b,
        hr.ctypes.data_as(_dp), hi.ctypes.data_as(_dp)))
    return hr + 1j * hi


def newfft_table(ktype: str, N: int, J: int, K: int, L: int, kb_alf=None, kb_m=None,
                 alpha=None, beta=None, phasing="real") -> np.ndarray:
    """Real table of newfft's interpolator `ktype` ('kb:minmax', 'kb:beatty',
    'diric', 'minmax:kb', 'minmax:unif', 'minmax:tuned', 'linear'; 'kb:user'
    with this dimension's kb_alf and integer kb_m; 'minmax:user' with its real
    alpha and beta; phasing 'real'), [J*L+1] (see mirt_newfft_ktype_table,
    mirt_newfft_kb_user_table, mirt_newfft_minmax_user_table); phasing
    'complex': the complex table (see mirt_newfft_table_complex)."""
    if phasing == "complex":
        return _newfft_table_complex(ktype, N, J, K, L, kb_alf, kb_m, alpha, beta)
    if phasing != "real":
        raise ValueError("phasing must be 'real' or 'complex'")
    h = np.empty(int(J) * int(L) + 1)
    lib = load()
    if ktype == "kb:user":
        a, m = _user_args(ktype, kb_alf, kb_m, alpha, beta)
        check(lib.mirt_newfft_kb_user_table(int(J), int(L), a, m, h.ctypes.data_as(_dp)))
    elif ktype == "minmax:user":
        a, b = _user_args(ktype, kb_alf, kb_m, alpha, beta)
        check(lib.mirt_newfft_minmax_user_table(int(N), int(J), int(K), int(L),
                                                a.ctypes.data_as(_dp), a.size, b,
                                                h.ctypes.data_as(_dp)))
    elif ktype in _KTYPES:
        check(lib.mirt_newfft_ktype_table(_KTYPES[ktype], int(N), int(J), int(K), int(L),
                                          h.ctypes.data_as(_dp)))
    else:
        raise ValueError(f"ktype must be one of {sorted(_KTYPES) + list(_USER_KTYPES)}")
    return h


def newfft_scale(ktype: str, N: int, J: int, K: int, nmid: float, kb_alf=None, kb_m=None,
                 alpha=None, beta=None) -> np.ndarray:
    """1D scaling factors of newfft's interpolator `ktype`, [N]."""
    s = np.empty(int(N))
    lib = load()
    if ktype == "kb:user":
        a, m = _user_args(ktype, kb_alf, kb_m, alpha, beta)
        check(lib.mirt_newfft_kb_user_scale(int(N), int(J), int(K), float(nmid), a, m,
                                            s.ctypes.data_as(_dp)))
    elif ktype == "minmax:user":
        a, b = _user_args(ktype, kb_alf, kb_m, alpha, beta)
        check(lib.mirt_newfft_minmax_user_scale(int(N), int(K), float(nmid),
                                                a.ctypes.data_as(_dp), a.size, b,
                                                s.ctypes.data_as(_dp)))
    elif ktype in _KTYPES:
        check(lib.mirt_newfft_ktype_scale(_KTYPES[ktype], int(N), int(J), int(K), float(nmid),
                                          s.ctypes.data_as(_dp)))
    else:
        raise ValueError(f"ktype must be one of {sorted(_KTYPES) + list(_USER_KTYPES)}")
    return s


def newfft_tables(ktype, Nd, Jd, Kd, Ld, phasing="real", kb_alf=None, kb_m=None, alpha=None,
                  beta=None):
    """The 1D tables and st.sn ([(Nd)] flattened, first index fastest) of
    newfft(..., 'ktype', ktype, 'phasing', phasing) in table mode, built in
    the library; user parameters per dimension (st.kb_alf(id), st.kb_m(id),
    st.alpha{id}, st.beta{id}: nufft/private/newfft_table_init.m:88-96).
    Nmid = floor(N/2) for phasing 'real', (N-1)/2 for 'complex'."""
    if phasing not in ("real", "complex"):
        raise ValueError("phasing must be 'real' or 'complex'")
    Nd = np.asarray(Nd)
    nmid = np.floor(Nd / 2) if phasing == "real" else (Nd - 1) / 2

    def user(d):
        pick = lambda v: None if v is None else v[d]
        return dict(kb_alf=pick(kb_alf), kb_m=pick(kb_m), alpha=pick(alpha), beta=pick(beta))
    D = len(Nd)
    tables = [newfft_table(ktype, Nd[d], Jd[d], Kd[d], Ld[d], phasing=phasing, **user(d))
              for d in range(D)]
    s = np.ones(1)
    for d in range(D):
        s = np.outer(s.ravel(order="F"), newfft_scale(ktype, Nd[d], Jd[d], Kd[d], float(nmid[d]),
                                                      **user(d)))
    return tables, s.ravel(order="F")


class NewfftPlan(NufftPlan):
    """st = newfft(om, Nd, 'Jd', Jd, 'Kd', Kd, 'n_shift', n_shift, 'mode',
    'table0' | 'table1', 'oversample', Ld, 'phasing', phasing) on the device
    (nufft/newfft.m, nufft/private/newfft_table_init.m).

    phasing 'real' (the reference's default) with ``tables=None`` builds the
    real tables and scaling factors of ``ktype`` in the library ('kb:minmax',
    the reference's default, 'kb:beatty', 'diric', 'minmax:kb', 'minmax:unif',
    'minmax:tuned', 'linear', 'kb:user' with per-dimension ``kb_alf`` and
    integer ``kb_m``, or 'minmax:user' with per-dimension ``alpha`` (lists of
    real coefficients) and ``beta``); with phasing 'complex' the complex
    tables of the same ktypes, with the scaling factors at Nmid = (N-1)/2; any
    other interpolator
    is given as ``tables`` (one 1D table per dimension, real or complex, J*L+1
    values) and ``sn`` ([(Nd)], first index fastest).
    phasing 'real' applies phase_before / phase_after with Nmid = floor(N/2);
    'complex' applies only exp(i om . n_shift) per sample.  Layouts and
    methods are those of NufftPlan.
    """

    def __init__(self, om, Nd, Jd=None, Kd=None, n_shift=None, mode="table1", Ld=None,
                 phasing="real", tables=None, sn=None, ncol=1, slice_moff=None, stream=None,
                 ktype="kb:minmax", kb_alf=None, kb_m=None, alpha=None, beta=None):
        om = np.asarray(om, dtype=np.float64)
        D = 1 if om.ndim == 1 else om.shape[1]
        Nd = _i32(Nd)
        Jd = _i32([6] * D if Jd is None else Jd)
        Kd = _i32(2 * Nd if Kd is None else Kd)
        if mode not in ("table0", "table1"):
            raise ValueError("mode must be 'table0' or 'table1'")
        if phasing not in ("real", "complex"):
            raise ValueError("phasing must be 'real' or 'complex'")
        self.order = 0 if mode == "table0" else 1
        if Ld is None:
            Ld = 2 ** 11 if self.order == 0 else 2 ** 9
        Ld = _i32(Ld if np.ndim(Ld) else [Ld] * D)
        self.phasing = phasing
        self.Nmid = (np.floor(Nd / 2) if phasing == "real" else (Nd - 1) / 2).astype(np.float64)
        if tables is None:
            tables, sn = newfft_tables(ktype, Nd, Jd, Kd, Ld, phasing, kb_alf=kb_alf, kb_m=kb_m,
                                       alpha=alpha, beta=beta)
        if sn is None:
            raise ValueError("sn is required with caller tables")
        self._tab = [np.ascontiguousarray(t) for t in tables]
        self._sn = np.asarray(sn).ravel(order="F")
        super().__init__(om, Nd, Jd, Kd, n_shift=n_shift, Ld=Ld, ncol=ncol,
                         slice_moff=slice_moff, stream=stream)

    def _create(self, omf, mo, stream):
        D = self.D
        cx = any(np.iscomplexobj(t) for t in self._tab)
        hr = [np.ascontiguousarray(np.real(t), dtype=np.float64) for t in self._tab]
        hi = [np.ascontiguousarray(np.imag(t), dtype=np.float64) for t in self._tab]
        for d in range(D):
            if hr[d].size != int(self.Jd[d]) * int(self.Ld[d]) + 1:
                raise ValueError(f"table {d} must have J*L+1 values")
        if self._sn.size != int(np.prod(self.Nd)):
            raise ValueError("sn must have prod(Nd) values")
        hr_p = (_dp * D)(*[t.ctypes.data_as(_dp) for t in hr])
        hi_p = (_dp * D)(*[t.ctypes.data_as(_dp) for t in hi]) if cx else None
        snr = np.ascontiguousarray(self._sn.real, dtype=np.float64)
        sni = np.ascontiguousarray(self._sn.imag, dtype=np.float64)
        nmid = np.ascontiguousarray(self.Nmid)
        h = C.c_void_p()
        check(self.lib.mirt_newfft_create(
            C.byref(h), D, self.Nd.ctypes.data_as(_i32p), self.Kd.ctypes.data_as(_i32p),
            self.Jd.ctypes.data_as(_i32p), self.Ld.ctypes.data_as(_i32p), hr_p, hi_p,
            self.order, snr.ctypes.data_as(_dp), sni.ctypes.data_as(_dp),
            nmid.ctypes.data_as(_dp) if self.phasing == "real" else None,
            self.n_shift.ctypes.data_as(_dp), omf.ctypes.data_as(_dp), self.Mtot,
            None if mo is None else mo.ctypes.data_as(_i64p), self.nslice, self.ncol,
            _stream_ptr(stream)))
        return h

    def fft(self, x):
        """X = st.fft(x) for a numpy image x[n1, n2, ...] (one column)."""
        return nufft(x, self)

    def adj(self, X):
        """x = st.adj(X) for numpy samples X[M] (one column)."""
        return nufft_adj(X, self)


def newfft(om, Nd, **kw) -> NewfftPlan:
    """st = newfft(om, Nd, 'Jd', ..., 'Kd', ..., 'n_shift', ..., 'mode', ...,
    'oversample', ..., 'phasing', ...) in table mode; see NewfftPlan."""
    if "oversample" in kw:
        kw["Ld"] = kw.pop("oversample")
    return NewfftPlan(om, Nd, **kw)


# ---------------------------------------------------------------------------
# MATLAB-style interface
# ---------------------------------------------------------------------------
_NUFFT_KTYPES = {"kaiser": 0, "minmax:kb": 3, "uniform": 4, "minmax:tuned": 5, "linear": 6,
                 "minmax:user": 8}


def _nufft_ktype_call(fn, ktype, N, J, K, L, params, out_len):
    code = _NUFFT_KTYPES.get(ktype)
    if code is None:
        raise ValueError(f"ktype must be one of {sorted(_NUFFT_KTYPES)}")
    kb_alf, kb_m, al, beta = 0.0, 0, None, 0.0
    if ktype == "kaiser" and params:
        code, kb_alf, kb_m = 7, float(params[0]), int(params[1])
        if float(params[1]) != kb_m:
            raise ValueError("kaiser: m must be an integer")
    elif ktype == "minmax:user":
        if len(params) != 2:
            raise ValueError("user must provide alpha/beta")
        al = np.ascontiguousarray(np.atleast_1d(np.asarray(params[0], dtype=np.float64)))
        beta = float(params[1])
    re, im = np.empty(out_len), np.empty(out_len)
    args = [code, int(N), int(J), int(K)] + ([int(L)] if L is not None else [])
    check(fn(*args, kb_alf, kb_m, None if al is None else al.ctypes.data_as(_dp),
             0 if al is None else al.size, beta, re.ctypes.data_as(_dp), im.ctypes.data_as(_dp)))
    return re + 1j * im


def nufft_table(ktype, N, J, K, L, *params) -> np.ndarray:
    """1D table of nufft_init(..., 'table', L, ktype, params...) (see
    mirt_nufft_ktype_table): [J*L+1] complex.  params: 'kaiser' [alpha, m]
    of this dimension, 'minmax:user' alpha (list), beta."""
    return _nufft_ktype_call(load().mirt_nufft_ktype_table, ktype, N, J, K, L, params,
                             int(J) * int(L) + 1)


def nufft_scale(ktype, N, J, K, *params) -> np.ndarray:
    """The 1D factors whose outer product is nufft_init's st.sn, [N] complex."""
    return _nufft_ktype_call(load().mirt_nufft_ktype_scale, ktype, N, J, K, None, params, int(N))


def nufft_init(om, Nd, Jd, Kd, n_shift=None, *args, ncol=1, slice_moff=None, stream=None):
    """st = nufft_init(om, Nd, Jd, Kd, n_shift, 'table', Ld, ktype, ...).

    ktype 'minmax:kb' (the reference's default, nufft/nufft_init.m:83-85) runs
    the library's NUFFT plan with its fused FFT passes; 'kaiser' [, alpha_list,
    m_list], 'minmax:tuned', 'minmax:user', alpha_list, beta_list, 'uniform' and
    'linear' build nufft_init's tables and scaling factors in the library and
    run them through the newfft plan with phasing 'complex', which is the same
    nufft / nufft_adj (only the n_shift phase around the gather).  As
    nufft_table_init.m:86-97 requires, 'kaiser' with parameters must use the
    same alpha and m in every dimension.
    """
    args = list(args)
    Ld = 1024
    if args and args[0] == "table":
        Ld = args[1] if len(args) > 1 else Ld
        rest = args[2:]
    else:
        rest = args
    ktype = rest[0] if rest else "minmax:kb"
    params = rest[1:]
    Nd = _i32(Nd)
    D = len(Nd)
    Jd, Kd = _i32(Jd), _i32(Kd)
    Ld = _i32(Ld if np.ndim(Ld) else [Ld] * D)
    if ktype == "minmax:kb":
        if params:
            raise ValueError("minmax:kb takes no parameters")
        return NufftPlan(om, Nd, Jd, Kd, n_shift=n_shift, Ld=Ld, ncol=ncol,
                         slice_moff=slice_moff, stream=stream)
    tables, sn = nufft_init_tables(ktype, Nd, Jd, Kd, Ld, *params)
    return NewfftPlan(om, Nd, Jd, Kd, n_shift=n_shift, mode="table0", Ld=Ld, phasing="complex",
                      tables=tables, sn=sn, ncol=ncol, slice_moff=slice_moff, stream=stream)


def nufft_init_tables(ktype, Nd, Jd, Kd, Ld, *params):
    """The 1D tables and st.sn ([(Nd)] flattened, first index fastest) of
    nufft_init(..., 'table', Ld, ktype, params...) for the interpolators
    other than 'minmax:kb', built in the library (params per dimension)."""
    Nd, Jd, Kd = _i32(Nd), _i32(Jd), _i32(Kd)
    D = len(Nd)
    Ld = _i32(Ld if np.ndim(Ld) else [Ld] * D)
    if ktype not in _NUFFT_KTYPES:
        raise ValueError(f"unknown kernel type {ktype!r}")
    if ktype == "kaiser" and params:
        if len(params) != 2:
            raise ValueError("kaiser should have no arguments, or both alpha and m")
        a, m = np.atleast_1d(params[0]), np.atleast_1d(params[1])
        if len(a) != D or len(m) != D:
            raise ValueError(f"#alpha={len(a)} #m={len(m)} vs dd={D}")
        if np.any(a != a[0]) or np.any(m != m[0]):
            raise ValueError("table based needs identical interpolator for each dimension")
        per_dim = [(a[d], m[d]) for d in range(D)]
    elif ktype == "minmax:user":
        if len(params) != 2:
            raise ValueError("user must provide alpha/beta")
        if len(params[0]) != D or len(params[1]) != D:
            raise ValueError("alpha/beta size mismatch")
        per_dim = [(params[0][d], params[1][d]) for d in range(D)]
    else:
        if params:
            raise ValueError(f"{ktype} takes no parameters")
        per_dim = [()] * D
    tables = [nufft_table(ktype, Nd[d], Jd[d], Kd[d], Ld[d], *per_dim[d]) for d in range(D)]
    s = np.ones(1, dtype=np.complex128)
    for d in range(D):
        s = np.outer(s.ravel(order="F"), nufft_scale(ktype, Nd[d], Jd[d], Kd[d], *per_dim[d]))
    return tables, s.ravel(order="F")


def _to_device_image(x, D, ncol):
    torch = _torch()
    x = np.asarray(x, dtype=np.complex64)
    if x.ndim == D:
        x = x[..., None]
    axes = tuple(range(D - 1, -1, -1)) + (D,)
    return torch.from_numpy(np.ascontiguousarray(np.transpose(x, axes))[None]).cuda()


def nufft(x, st: NufftPlan):
    """X = nufft(x, st) for a numpy image x[n1, n2, ...] (one column)."""
    xd = _to_device_image(x, st.D, st.ncol)
    X = st.forward(xd)
    return X.cpu().numpy()[:, 0].astype(np.complex128)


def nufft_adj(X, st: NufftPlan):
    """x = nufft_adj(X, st) for numpy samples X[M] (one column)."""
    torch = _torch()
    Xd = torch.from_numpy(np.asarray(X, dtype=np.complex64).reshape(-1, 1).copy()).cuda()
    x = st.adjoint(Xd).cpu().numpy()[0, ..., 0]
    return np.transpose(x, tuple(range(st.D - 1, -1, -1))).astype(np.complex128)


class NufftGraph:
    """One captured batched NUFFT step (mirt_nufft_capture); keeps its plan and
    buffers alive."""

    def __init__(self, plan, x, X, xa):
        self.plan, self.bufs, self.lib = plan, (x, X, xa), plan.lib
        h = C.c_void_p()
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        check(self.lib.mirt_nufft_capture(plan.handle, ptr(x), ptr(X), ptr(xa), C.byref(h)))
        self.handle = h

    def launch(self, stream=None):
        check(self.lib.mirt_graph_launch(self.handle, _stream_ptr(stream)))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mirt_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
