"""CPU: the C-ABI library loads, exports every declared symbol, builds its
FP64 tables like the oracle, and rejects bad arguments with the reference
gateways' messages (no GPU work is started by any of these calls)."""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

import mirt_b200 as mb
from mirt_b200 import _lib
from oracle import nufft_ref as nr
from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "mirt_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mirt_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    lib = mb.load()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.exported_names())


def test_version():
    assert mb.load().mirt_version() >= 100


@pytest.mark.parametrize("N,J,K,L", [(64, 6, 128, 1024), (256, 6, 512, 1024),
                                     (128, 6, 256, 512), (60, 5, 120, 64), (30, 4, 64, 32)])
def test_tables_match_oracle(N, J, K, L):
    h = mb.minmax_kb_table(N, J, K, L)
    ho = nr.table_1d(N, J, K, L)
    assert np.abs(h - ho).max() <= 1e-10 * np.abs(ho).max()
    s = mb.minmax_kb_scale(N, J, K)
    a, b = nr.nufft_alpha_kb_fit(N, J, K)
    so = nr.nufft_scale1(N, K, a, b)
    assert np.abs(s - so).max() <= 1e-12 * np.abs(so).max()


def _args2(**kw):
    a = dict(ck=np.zeros((8, 8), complex), h1=np.zeros(6 * 4 + 1), h2=np.zeros(6 * 4 + 1),
             J=np.array([6, 6], np.int32), L=np.array([4, 4], np.int32), tm=np.zeros((3, 2)))
    a.update(kw)
    return a


@pytest.mark.parametrize("kw,msg", [
    (dict(ck=np.zeros((8, 8))), "interp2_table_mex failed: mxIsComplexDouble"),
    (dict(J=np.array([6, 6, 6], np.int32)), "interp2_table_mex failed: J must be [1,2]"),
    (dict(J=np.array([6, 6], np.int64)), "interp2_table_mex failed: J must be [1,2]"),
    (dict(L=np.array([4], np.int32)), "interp2_table_mex failed: L must be [1,2]"),
    (dict(h1=np.zeros(6 * 4)), "interp2_table_mex failed: h1 size problem"),
    (dict(h2=np.zeros((6 * 4 + 1, 2))), "interp2_table_mex failed: h2 size problem"),
    (dict(tm=np.zeros((3, 3))), "interp2_table_mex failed: tm must have 2 columns"),
    (dict(h1=np.zeros(25, complex)), "h must be real or complex double (preferably real)"),
])
def test_interp2_argument_errors(kw, msg):
    with pytest.raises(mb.MexError, match=re.escape(msg)):
        mb.interp2_table_mex(**_args2(**kw))


def test_order_and_flip_errors():
    a = _args2(h1=np.zeros(25, complex), h2=np.zeros(25, complex))
    with pytest.raises(mb.MexError, match="only 0th order implemented for complex"):
        mb.interp2_table_mex(**a, order=np.array([1], np.int32))
    with pytest.raises(mb.MexError, match="bad order"):
        mb.interp2_table_mex(**_args2(), order=np.array([2], np.int32))
    with pytest.raises(mb.MexError, match="flip not compiled"):
        mb.interp2_table_mex(**_args2(), order=np.array([0], np.int32),
                             flips=np.array([1, 0], np.int32))
    with pytest.raises(mb.MexError, match=re.escape("order must be scalar int32 (0 | 1)")):
        mb.interp2_table_mex(**_args2(), order=np.array([0, 1], np.int32))


def test_adjoint_and_1d_3d_errors():
    h = np.zeros(25)
    J2, L2, K2 = (np.array([6, 6], np.int32), np.array([4, 4], np.int32),
                  np.array([8, 8], np.int32))
    with pytest.raises(mb.MexError, match=re.escape("interp2_table_adj_mex() failed: t_m must be Mx2 matrix")):
        mb.interp2_table_adj_mex(np.zeros((3, 1), complex), h, h, J2, L2, np.zeros((4, 2)), K2)
    with pytest.raises(mb.MexError, match=re.escape("interp2_table_adj_mex() failed: K must be int32 [1,2]")):
        mb.interp2_table_adj_mex(np.zeros((3, 1), complex), h, h, J2, L2, np.zeros((3, 2)),
                                 np.array([8], np.int32))
    J1, L1 = np.array([6], np.int32), np.array([4], np.int32)
    with pytest.raises(mb.MexError, match=re.escape("interp1_table_mex() failed: t_m must be col vector.")):
        mb.interp1_table_mex(np.zeros((8, 1), complex), h, J1, L1, np.zeros((3, 2)))
    with pytest.raises(mb.MexError, match=re.escape("interp1_table_adj_mex() failed: h must be col vector")):
        mb.interp1_table_adj_mex(np.zeros((3, 1), complex), np.zeros((25, 2)), J1, L1,
                                 np.zeros((3, 1)), np.array([8], np.int32))
    J3, L3 = np.array([6, 6, 6], np.int32), np.array([4, 4, 4], np.int32)
    with pytest.raises(mb.MexError, match=re.escape("interp3_table_mex failed: h3 size problem")):
        mb.interp3_table_mex(np.zeros((8, 8, 8), complex), h, h, np.zeros(3), J3, L3,
                             np.zeros((3, 3)))
    with pytest.raises(mb.MexError, match=re.escape("interp3_table_adj_mex() failed: L must be int32 [1,3]")):
        mb.interp3_table_adj_mex(np.zeros((3, 1), complex), h, h, h, J3, L2, np.zeros((3, 3)),
                                 np.array([8, 8, 8], np.int32))


def test_4d_gateway_errors():
    """interp4_table_mex.c:43-98 and interp4_table_adj_mex.c:46-104: the checks
    in order, with the gateways' texts (the forward one fails as
    interp3_table_mex, as the reference's own gateway does)."""
    h = np.zeros(25)
    J4, L4, K4 = (np.array([6, 6, 6, 6], np.int32), np.array([4, 4, 4, 4], np.int32),
                  np.array([8, 8, 8, 8], np.int32))
    ck = np.zeros((8, 8, 8, 8), complex)
    tm = np.zeros((3, 4))
    fm = np.zeros((3, 1), complex)
    f = "interp3_table_mex failed: "
    with pytest.raises(mb.MexError, match=re.escape(f + "mxIsComplexDouble")):
        mb.interp4_table_mex(ck.real, h, h, h, h, J4, L4, tm)
    with pytest.raises(mb.MexError, match=re.escape(f + "J must be [1,4]")):
        mb.interp4_table_mex(ck, h, h, h, h, J4[:3], L4, tm)
    with pytest.raises(mb.MexError, match=re.escape(f + "L must be [1,4]")):
        mb.interp4_table_mex(ck, h, h, h, h, J4, L4[:2], tm)
    with pytest.raises(mb.MexError, match=re.escape(f + "flips must be [1 4] int32 (0 | 1)")):
        mb.interp4_table_mex(ck, h, h, h, h, J4, L4, tm, flips=np.zeros(3, np.int32))
    with pytest.raises(mb.MexError, match=re.escape(f + "h4 size problem")):
        mb.interp4_table_mex(ck, h, h, h, np.zeros(24), J4, L4, tm)
    with pytest.raises(mb.MexError, match=re.escape(f + "tm must have 4 columns")):
        mb.interp4_table_mex(ck, h, h, h, h, J4, L4, np.zeros((3, 3)))
    with pytest.raises(mb.MexError, match=re.escape(f + "flip not compiled")):
        mb.interp4_table_mex(ck, h, h, h, h, J4, L4, tm, flips=np.array([0, 0, 0, 1], np.int32))
    with pytest.raises(mb.MexError, match="h must be real or complex double"):
        mb.interp4_table_mex(ck, h, h, h, np.zeros(25, complex), J4, L4, tm)
    a = "interp4_table_adj_mex() failed: "
    with pytest.raises(mb.MexError, match=re.escape(a + "K must be int32 [1,4]")):
        mb.interp4_table_adj_mex(fm, h, h, h, h, J4, L4, tm, K4[:3])
    with pytest.raises(mb.MexError, match=re.escape(a + "h2 size problem")):
        mb.interp4_table_adj_mex(fm, h, np.zeros((25, 2)), h, h, J4, L4, tm, K4)
    with pytest.raises(mb.MexError, match=re.escape(a + "t_m must be Mx4 matrix")):
        mb.interp4_table_adj_mex(fm, h, h, h, h, J4, L4, np.zeros((4, 4)), K4)
    with pytest.raises(mb.MexError, match=re.escape(a + "only 0th order implemented for complex")):
        hc = np.zeros(25, complex)
        mb.interp4_table_adj_mex(fm, hc, hc, hc, hc, J4, L4, tm, K4, order=np.ones(1, np.int32))


def test_j_larger_than_k_is_refused():
    """The GPU kernels wrap each tap once, so J > K is refused before any
    device work (the 4th dimension of the 4D gateways wraps on the host)."""
    h = np.zeros(25)
    with pytest.raises(mb.MexError, match="J larger than K is not supported"):
        mb.interp2_table_mex(np.zeros((8, 4), complex), h, h, np.array([6, 6], np.int32),
                             np.array([4, 4], np.int32), np.zeros((3, 2)))
    with pytest.raises(mb.MexError, match="J larger than K is not supported"):
        mb.interp4_table_adj_mex(np.zeros((3, 1), complex), h, h, h, h,
                                 np.array([6, 6, 6, 6], np.int32), np.array([4, 4, 4, 4], np.int32),
                                 np.zeros((3, 4)), np.array([8, 5, 8, 2], np.int32))


def test_valid_call_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mb.MirtError, match="no CUDA device"):
        mb.interp2_table_mex(**_args2())


def test_plan_setters_reject_null_plans():
    """The spread / gather selectors, the fault read-out and the newfft
    constructor check their pointers before touching a device."""
    import ctypes as C
    lib = _lib.load()
    assert lib.mirt_interp_plan_set_sweep(None, 1, 1) == 1
    assert "plan is NULL" in lib.mirt_last_error().decode()
    assert lib.mirt_interp_plan_set_gather(None, 1) == 1
    f = C.c_int32(7)
    assert lib.mirt_interp_plan_fault(None, C.byref(f)) == 1
    assert lib.mirt_interp_plan_set_deterministic(None, 1) == 1
    assert lib.mirt_newfft_create(None, 2, None, None, None, None, None, None, 1, None, None, None,
                                  None, None, 0, None, 1, 1, None) == 1
    assert "output pointer is NULL" in lib.mirt_last_error().decode()


def test_header_builds_and_links_from_c99(tmp_path):
    """The boundary as a mex gateway sees it: a strict C99 program includes
    include/mirt_b200.h, links libmirt_b200.so and makes calls that need no
    GPU (the version, a gateway argument error with its text)."""
    import os
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "mirt_b200")
    src = tmp_path / "gateway_check.c"
    src.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "mirt_b200.h"\n'
        "int main(void) {\n"
        "  int32_t J[2] = {6, 6}, L[2] = {4, 4};\n"
        "  if (mirt_version() < 1) return 2;\n"
        "  int rc = mirt_interp2_table_mex(NULL, NULL, NULL, 0, NULL, NULL, 0, 0, NULL, NULL, 0, 0,\n"
        "                                  J, 2, L, 2, NULL, 0, 0, NULL, 0, NULL, 0, NULL, NULL);\n"
        "  printf(\"%d %s\\n\", rc, mirt_last_error());\n"
        "  return rc == MIRT_ERR_ARG && strstr(mirt_last_error(), \"mxIsComplexDouble\") ? 0 : 3;\n"
        "}\n")
    exe = tmp_path / "gateway_check"
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic",
                         "-I" + os.path.join(root, "include"), str(src), "-o", str(exe),
                         "-L" + libdir, "-lmirt_b200", "-Wl,-rpath," + libdir],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "interp2_table_mex failed: mxIsComplexDouble" in run.stdout


def _plan_create(D, K, J, L, tabs, order=0, M=3, moff=None, nslice=1, ncol=2, cplx=False):
    import ctypes as C
    lib = _lib.load()
    K, J, L = (np.asarray(v, dtype=np.int32) for v in (K, J, L))
    keep = [np.ascontiguousarray(t, dtype=np.float64) if t is not None else None for t in tabs]
    dp = C.POINTER(C.c_double)
    hr = (dp * max(D, 1))(*[t.ctypes.data_as(dp) if t is not None else dp() for t in keep])
    hi = (dp * max(D, 1))(*[t.ctypes.data_as(dp) if t is not None else dp() for t in keep]) \
        if cplx else None
    tm = np.zeros(M * D)
    mo = None if moff is None else np.asarray(moff, dtype=np.int64)
    h = C.c_void_p()
    i32p, i64p = C.POINTER(C.c_int32), C.POINTER(C.c_int64)
    rc = lib.mirt_interp_plan_create(
        C.byref(h), D, K.ctypes.data_as(i32p), J.ctypes.data_as(i32p), L.ctypes.data_as(i32p),
        hr, hi, order, tm.ctypes.data_as(dp), M, None if mo is None else mo.ctypes.data_as(i64p),
        nslice, ncol, None, None, None)
    return rc, lib.mirt_last_error().decode()


def test_plan_arguments_checked_before_the_device():
    """mirt_interp_plan_create refuses bad arguments with their own message,
    before it looks for a device (here: none)."""
    t = np.zeros(6 * 4 + 1)
    cases = [
        (dict(D=5, K=[8] * 5, J=[6] * 5, L=[4] * 5, tabs=[t] * 5), "D must be 1, 2, 3 or 4"),
        (dict(D=2, K=[8, 5], J=[6, 6], L=[4, 4], tabs=[t, t]), "J must not exceed K"),
        (dict(D=4, K=[8, 8, 8, 3], J=[6, 6, 6, 17], L=[4] * 4, tabs=[t] * 3 + [np.zeros(69)]),
         "J must be in 1..16"),
        (dict(D=3, K=[8] * 3, J=[6] * 3, L=[4] * 3, tabs=[t, None, t]), "NULL table"),
        (dict(D=2, K=[8, 8], J=[6, 6], L=[4, 4], tabs=[t, t], order=1, cplx=True),
         "only 0th order implemented for complex"),
        (dict(D=2, K=[8, 8], J=[6, 6], L=[4, 4], tabs=[t, t], moff=[0, 1, 2], nslice=2),
         "slice offsets must start at 0 and end at Mtot"),
        (dict(D=2, K=[8, 8], J=[6, 6], L=[4, 4], tabs=[t, t], nslice=2),
         "slice offsets required"),
    ]
    for kw, msg in cases:
        rc, err = _plan_create(**kw)
        assert rc == _lib.MIRT_ERR_ARG and msg in err, (kw, rc, err)
    import torch
    if not torch.cuda.is_available():
        # a 4D plan with K4 < J4 is valid: the 4th dimension wraps on the host
        rc, err = _plan_create(D=4, K=[8, 8, 8, 3], J=[6, 6, 6, 4], L=[4] * 4,
                               tabs=[t, t, t, np.zeros(17)])
        assert "no CUDA device" in err


@pytest.mark.parametrize("D", [1, 2, 3, 4])
def test_gateways_with_no_samples(D):
    """M = 0 samples: the adjoint returns the zero grid and the forward an empty
    fm, as the reference kernels do (interp2_table1_adj.c:57-58 clears ck
    before its sample loop); no device is needed for that."""
    h = np.zeros(6 * 4 + 1)
    J, L = np.full(D, 6, np.int32), np.full(D, 4, np.int32)
    K = np.full(D, 8, np.int32)
    tm = np.zeros((0, D))
    fm = np.zeros((0, 3), complex)
    hs = [h] * D
    adj = {1: mb.interp1_table_adj_mex, 2: mb.interp2_table_adj_mex, 3: mb.interp3_table_adj_mex,
           4: mb.interp4_table_adj_mex}[D]
    ck = adj(fm, *hs, J if D > 1 else J[:1], L if D > 1 else L[:1], tm, K if D > 1 else K[:1])
    assert ck.shape == (8 ** D, 3) and not ck.any()
    fwd = {1: mb.interp1_table_mex, 2: mb.interp2_table_mex, 3: mb.interp3_table_mex,
           4: mb.interp4_table_mex}[D]
    grid = np.ones((8,) * D + ((2,) if D > 1 else ()), complex)
    if D == 1:
        grid = np.ones((8, 2), complex)
    out = fwd(grid, *hs, J, L, tm)
    assert out.shape == (0, 2)
