"""ctypes binding of libmirt_b200.so (the C ABI of include/mirt_b200.h).

The library is built in-tree by ``python -m mirt_b200.build``.  Loading fails
loudly when it is missing: there is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmirt_b200.so")

MIRT_OK = 0
MIRT_ERR_ARG = 1
MIRT_ERR_CUDA = 2
MIRT_ERR_ALLOC = 3
MIRT_ERR_FFT = 4


class MirtError(RuntimeError):
    """A libmirt_b200 call returned an error code."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64

# argument lists of every exported function (must match include/mirt_b200.h)
_TAB = [_dp, _dp, _i64, _i64]                     # re, im, rows, cols
_INTS = [_i32p, _i64]                             # data, numel
_SIGS = {
    "mirt_last_error": ([], C.c_char_p),
    "mirt_version": ([], C.c_int),
    "mirt_interp1_table_mex": ([_dp, _dp, _i64, _i64] + _TAB + _INTS * 2 + [_dp, _i64, _i64]
                               + _INTS * 2 + [_dp, _dp], C.c_int),
    "mirt_interp2_table_mex": ([_dp, _dp, _i64p, _i32] + _TAB * 2 + _INTS * 2 + [_dp, _i64, _i64]
                               + _INTS * 2 + [_dp, _dp], C.c_int),
    "mirt_interp3_table_mex": ([_dp, _dp, _i64p, _i32] + _TAB * 3 + _INTS * 2 + [_dp, _i64, _i64]
                               + _INTS * 2 + [_dp, _dp], C.c_int),
    "mirt_interp4_table_mex": ([_dp, _dp, _i64p, _i32] + _TAB * 4 + _INTS * 2 + [_dp, _i64, _i64]
                               + _INTS * 2 + [_dp, _dp], C.c_int),
    "mirt_interp1_table_adj_mex": ([_dp, _dp, _i64, _i64] + _TAB + _INTS * 2
                                   + [_dp, _i64, _i64] + _INTS * 3 + [_dp, _dp], C.c_int),
    "mirt_interp2_table_adj_mex": ([_dp, _dp, _i64, _i64] + _TAB * 2 + _INTS * 2
                                   + [_dp, _i64, _i64] + _INTS * 3 + [_dp, _dp], C.c_int),
    "mirt_interp3_table_adj_mex": ([_dp, _dp, _i64, _i64] + _TAB * 3 + _INTS * 2
                                   + [_dp, _i64, _i64] + _INTS * 3 + [_dp, _dp], C.c_int),
    "mirt_interp4_table_adj_mex": ([_dp, _dp, _i64, _i64] + _TAB * 4 + _INTS * 2
                                   + [_dp, _i64, _i64] + _INTS * 3 + [_dp, _dp], C.c_int),
    "mirt_interp_plan_create": ([C.POINTER(_vp), _i32, _i32p, _i32p, _i32p,
                                 C.POINTER(_dp), C.POINTER(_dp), _i32, _dp, _i64, _i64p, _i32,
                                 _i32, _dp, _dp, _vp], C.c_int),
    "mirt_interp_plan_forward": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_interp_plan_adjoint": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_interp_plan_autotune": ([_vp, _vp], C.c_int),
    "mirt_interp_plan_config": ([_vp, _i32p, _i32], C.c_int),
    "mirt_interp_plan_set_spread": ([_vp, _i32p, _i32, _i32, _vp], C.c_int),
    "mirt_interp_plan_set_deterministic": ([_vp, _i32], C.c_int),
    "mirt_interp_plan_set_ownership": ([_vp, _i32, _vp], C.c_int),
    "mirt_interp_plan_set_sweep": ([_vp, _i32, _i32], C.c_int),
    "mirt_interp_plan_set_gather": ([_vp, _i32], C.c_int),
    "mirt_interp_plan_fault": ([_vp, _i32p], C.c_int),
    "mirt_interp_plan_set_fault_test": ([_vp, _i32], C.c_int),
    "mirt_interp_plan_set_dense": ([_vp, _i32], C.c_int),
    "mirt_interp_plan_set_staged": ([_vp, _i32], C.c_int),
    "mirt_dcf_pipe": ([_vp, _vp, _i32, _i32, C.c_double, _dp, _i32p, _dp, _vp], C.c_int),
    "mirt_dcf_jackson": ([_vp, _vp, _vp], C.c_int),
    "mirt_dcf_scale": ([_vp, _vp, _dp, _vp], C.c_int),
    "mirt_nufft_capture": ([_vp, _vp, _vp, _vp, C.POINTER(_vp)], C.c_int),
    "mirt_graph_launch": ([_vp, _vp], C.c_int),
    "mirt_graph_destroy": ([_vp], C.c_int),
    "mirt_sense_create": ([C.POINTER(_vp), _vp, _vp, _dp, _vp], C.c_int),
    "mirt_sense_forward": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_sense_adjoint": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_sense_reg": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_sense_cg": ([_vp, _vp, _vp, _vp, _i32, _vp, _dp, C.POINTER(C.c_float), _vp], C.c_int),
    "mirt_sense_warm_start": ([_vp, _vp, _vp, _vp, _vp], C.c_int),
    "mirt_sense_destroy": ([_vp], C.c_int),
    "mirt_sense_toeplitz": ([_vp, _dp, _vp], C.c_int),
    "mirt_sense_precon_dcf": ([_vp, _dp, _vp, C.c_double, _vp], C.c_int),
    "mirt_sense_pcg": ([_vp, _vp, _vp, _vp, _i32, _i32, _vp, _dp, C.POINTER(C.c_float), _vp],
                       C.c_int),
    "mirt_toeplitz_create": ([C.POINTER(_vp), _dp, _i64, _i64p, _i32, _i32p, _i32p, _i32p,
                              _i32p, _vp, _i32, _vp], C.c_int),
    "mirt_toeplitz_apply": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_toeplitz_destroy": ([_vp], C.c_int),
    "mirt_dcf_features": ([_vp, _i64, _i64p, _i32, _i32p, _vp, _vp], C.c_int),
    "mirt_mlp_create": ([C.POINTER(_vp), C.POINTER(C.c_float)], C.c_int),
    "mirt_mlp_params": ([_vp, C.POINTER(C.c_float)], C.c_int),
    "mirt_mlp_grad": ([_vp, _vp, _vp, _i64, C.POINTER(C.c_float), C.POINTER(C.c_float), _vp],
                      C.c_int),
    "mirt_mlp_train": ([_vp, _vp, _vp, _i64, _i32, _i32, C.c_float, C.c_uint64,
                        C.POINTER(C.c_float), _vp], C.c_int),
    "mirt_mlp_infer": ([_vp, _vp, _i64, C.c_float, C.c_float, _vp, _vp, _vp], C.c_int),
    "mirt_mlp_set_tensor_cores": ([_vp, _i32], C.c_int),
    "mirt_mlp_destroy": ([_vp], C.c_int),
    "mirt_interp_plan_destroy": ([_vp], C.c_int),
    "mirt_nufft_create": ([C.POINTER(_vp), _i32, _i32p, _i32p, _i32p, _i32p, _dp, _dp, _i64,
                           _i64p, _i32, _i32, _vp], C.c_int),
    "mirt_nufft_forward": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_nufft_adjoint": ([_vp, _vp, _vp, _vp], C.c_int),
    "mirt_nufft_forward_host": ([_vp, _fp, _fp, _vp], C.c_int),
    "mirt_nufft_adjoint_host": ([_vp, _fp, _fp, _vp], C.c_int),
    "mirt_nufft_interp_plan": ([_vp], _vp),
    "mirt_nufft_autotune": ([_vp, _vp], C.c_int),
    "mirt_nufft_config": ([_vp, _i32p, _i32], C.c_int),
    "mirt_nufft_destroy": ([_vp], C.c_int),
    "mirt_interp_gather_noalloc": ([_i32, _i32p, _i32p, _i32p, C.POINTER(_vp), _i32, _i32, _dp,
                                    _i64, _i32, _vp, _vp, _vp], C.c_int),
    "mirt_minmax_kb_table": ([_i32, _i32, _i32, _i32, _dp, _dp], C.c_int),
    "mirt_minmax_kb_scale": ([_i32, _i32, _i32, _dp, _dp], C.c_int),
    "mirt_newfft_create": ([C.POINTER(_vp), _i32, _i32p, _i32p, _i32p, _i32p, C.POINTER(_dp),
                            C.POINTER(_dp), _i32, _dp, _dp, _dp, _dp, _dp, _i64, _i64p, _i32,
                            _i32, _vp], C.c_int),
    "mirt_newfft_kb_table": ([_i32, _i32, _dp], C.c_int),
    "mirt_newfft_kb_scale": ([_i32, _i32, _i32, C.c_double, _dp], C.c_int),
    "mirt_newfft_ktype_table": ([_i32, _i32, _i32, _i32, _i32, _dp], C.c_int),
    "mirt_newfft_ktype_scale": ([_i32, _i32, _i32, _i32, C.c_double, _dp], C.c_int),
    "mirt_nufft_ktype_table": ([_i32, _i32, _i32, _i32, _i32, C.c_double, _i32, _dp, _i32,
                                C.c_double, _dp, _dp], C.c_int),
    "mirt_nufft_ktype_scale": ([_i32, _i32, _i32, _i32, C.c_double, _i32, _dp, _i32,
                                C.c_double, _dp, _dp], C.c_int),
    "mirt_newfft_table_complex": ([_i32, _i32, _i32, _i32, _i32, C.c_double, _i32, _dp, _i32,
                                   C.c_double, _dp, _dp], C.c_int),
    "mirt_newfft_kb_user_table": ([_i32, _i32, C.c_double, _i32, _dp], C.c_int),
    "mirt_newfft_kb_user_scale": ([_i32, _i32, _i32, C.c_double, C.c_double, _i32, _dp],
                                  C.c_int),
    "mirt_newfft_minmax_user_table": ([_i32, _i32, _i32, _i32, _dp, _i32, C.c_double, _dp],
                                      C.c_int),
    "mirt_newfft_minmax_user_scale": ([_i32, _i32, C.c_double, _dp, _i32, C.c_double, _dp],
                                      C.c_int),
}

_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Load libmirt_b200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mirt_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def exported_names() -> list[str]:
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != MIRT_OK:
        msg = load().mirt_last_error().decode(errors="replace")
        raise MirtError(rc, msg)
