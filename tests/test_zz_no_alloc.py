"""GPU: the gather entry point that allocates no device memory.

mirt_interp_gather_noalloc serves callers that cannot call cudaMalloc (code
running under CUDA-graph stream capture, hosts whose device memory belongs to
their own pool, real-time loops).  Its scratch is a fixed array inside the
library, so these checks call it through the C ABI on caller-owned torch
buffers and compare it with the plan-based gather (mirt_interp_plan_forward)
on two calls in a row -- the second on a different trajectory and grid, so a
stale scratch from the first call would show -- and check that a sample count
beyond the fixed scratch is refused.

This file is collected last on purpose: a failure here leaves every other test
already run.  It also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import mirt_b200 as mb
from mirt_b200._lib import MIRT_ERR_ARG, MIRT_OK, load
from conftest import rel_l2

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-6


def _i32(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


def _noalloc_gather(K, J, L, tabs_dev, tm, ck_dev, ncol, torch, real_tab=0, order=0):
    lib = load()
    D = len(K)
    Ka, Ja, La = _i32(K), _i32(J), _i32(L)
    tab_ptrs = (C.c_void_p * D)(*[C.c_void_p(t.data_ptr()) for t in tabs_dev])
    tm_dev = torch.from_numpy(np.ascontiguousarray(tm.T)).cuda()   # [D][M] = column-major [M, D]
    M = tm.shape[0]
    fm = torch.empty((M, ncol), dtype=torch.complex64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.mirt_interp_gather_noalloc(
        D, Ka.ctypes.data_as(C.POINTER(C.c_int32)), Ja.ctypes.data_as(C.POINTER(C.c_int32)),
        La.ctypes.data_as(C.POINTER(C.c_int32)), tab_ptrs, int(real_tab), int(order),
        C.cast(C.c_void_p(tm_dev.data_ptr()), C.POINTER(C.c_double)), M, ncol,
        C.c_void_p(ck_dev.data_ptr()), C.c_void_p(fm.data_ptr()), stream)
    assert rc == MIRT_OK, lib.mirt_last_error().decode()
    torch.cuda.synchronize()
    return fm.cpu().numpy()


def _case(seed, K, N, nspoke, nread, ncol, torch):
    rng = np.random.default_rng(seed)
    J, L = [6, 6], [1024, 1024]
    tabs = [mb.minmax_kb_table(N, 6, K[0], 1024), mb.minmax_kb_table(N, 6, K[1], 1024)]
    r = np.linspace(-np.pi, np.pi, nread, endpoint=False)
    ang = np.arange(nspoke) * np.pi / nspoke + rng.uniform(0, 0.1)
    om = np.stack([np.outer(np.cos(ang), r).ravel(), np.outer(np.sin(ang), r).ravel()], 1)
    tm = np.stack([om[:, d] / (2 * np.pi / K[d]) for d in range(2)], 1)
    plan = mb.InterpPlan(K, J, L, tabs, tm, ncol)
    ck = (rng.standard_normal(plan.grid_shape) + 1j * rng.standard_normal(plan.grid_shape))
    ck_dev = torch.from_numpy(ck.astype(np.complex64)).cuda()
    ref = plan.forward(ck_dev).cpu().numpy()
    plan.close()
    tabs_dev = [torch.from_numpy(t.astype(np.complex64)).cuda() for t in tabs]
    got = _noalloc_gather(K, J, L, tabs_dev, tm, ck_dev, ncol, torch)
    return got, ref


def test_noalloc_gather_matches_plan_twice():
    import torch
    # first call, then a second on another trajectory / grid / column count
    got1, ref1 = _case(1, [128, 128], 64, 64, 128, 4, torch)
    assert rel_l2(got1, ref1) <= FWD_TOL
    got2, ref2 = _case(2, [96, 80], 40, 40, 96, 32, torch)
    assert rel_l2(got2, ref2) <= FWD_TOL
    # and the first problem again after the second overwrote the scratch
    got3, ref3 = _case(1, [128, 128], 64, 64, 128, 4, torch)
    assert rel_l2(got3, ref3) <= FWD_TOL


def _refuses(D, M):
    """The size check runs before any pointer is used: dummy pointers suffice."""
    lib = load()
    K, J, L = _i32([512] * D), _i32([6] * D), _i32([1024] * D)
    dummy = (C.c_void_p * D)(*[C.c_void_p(16)] * D)
    rc = lib.mirt_interp_gather_noalloc(
        D, K.ctypes.data_as(C.POINTER(C.c_int32)), J.ctypes.data_as(C.POINTER(C.c_int32)),
        L.ctypes.data_as(C.POINTER(C.c_int32)), dummy, 0, 0,
        C.cast(C.c_void_p(16), C.POINTER(C.c_double)), M, 1, C.c_void_p(16),
        C.c_void_p(16), None)
    return rc == MIRT_ERR_ARG and "exceeds the fixed scratch" in lib.mirt_last_error().decode()


# floor((32 MiB - 256) / (8 * sum(J) + 16)): 112 bytes a sample in 2D, 160 in 3D (J = 6)
M_MAX_2D = (32 * 2 ** 20 - 256) // 112
M_MAX_3D = (32 * 2 ** 20 - 256) // 160


def test_noalloc_rejects_sizes_beyond_scratch():
    assert M_MAX_2D == 299_590 and M_MAX_3D == 209_713
    assert _refuses(2, 400_000)
    assert _refuses(2, M_MAX_2D + 1)
    assert _refuses(3, M_MAX_3D + 1)


def _oracle_case(D, K, J, L, tabs, tm, ncol, order, seed, torch):
    """noalloc gather vs the reference's FP64 kernels on one problem."""
    import oracle
    from conftest import ref_impl
    rng = np.random.default_rng(seed)
    nk = int(np.prod(K))
    ck = rng.standard_normal((nk, ncol)) + 1j * rng.standard_normal((nk, ncol))
    real = not any(np.iscomplexobj(t) for t in tabs)
    ref = oracle.interp_for(ck, tabs, J, L, tm, K, order, impl=ref_impl(), nthreads=8)
    # device grid [K_D]..[K_1][ncol]: column-major points, column innermost
    ck_dev = torch.from_numpy(np.ascontiguousarray(ck).astype(np.complex64)).cuda()
    tdt = np.float32 if real else np.complex64
    tabs_dev = [torch.from_numpy(np.asarray(t).astype(tdt)).cuda() for t in tabs]
    got = _noalloc_gather(K, J, L, tabs_dev, tm, ck_dev, ncol, torch, real_tab=int(real),
                          order=order)
    return got, ref


def test_noalloc_gather_3d_real_tables_and_ragged_columns():
    """The other kernel instantiations it reaches: 3D with J = 6 (160 bytes of
    scratch a sample), real tables of order 1, and ncol = 10 (coil groups of
    8 lanes with a partial second group), each against the oracle."""
    import torch
    rng = np.random.default_rng(70)
    # 3D, J = 6, complex min-max tables, 8 columns
    K, J, L = [32, 24, 20], [6, 6, 6], [512, 512, 512]
    tabs = [mb.minmax_kb_table(k // 2, 6, k, 512) for k in K]
    tm = rng.uniform(-40, 40, (5000, 3))
    got, ref = _oracle_case(3, K, J, L, tabs, tm, 8, 0, 71, torch)
    assert rel_l2(got, ref) <= FWD_TOL
    # 2D real tables, order 1 (newfft's table1 form), 3 columns
    K, J, L = [64, 48], [6, 6], [512, 512]
    tabs = [mb.newfft_kb_table(6, 512)] * 2
    tm = rng.uniform(-70, 70, (6000, 2))
    got, ref = _oracle_case(2, K, J, L, tabs, tm, 3, 1, 72, torch)
    assert rel_l2(got, ref) <= FWD_TOL
    # 2D complex tables, 10 columns
    K, J, L = [64, 64], [6, 6], [1024, 1024]
    tabs = [mb.minmax_kb_table(32, 6, 64, 1024)] * 2
    tm = rng.uniform(-64, 64, (4000, 2))
    got, ref = _oracle_case(2, K, J, L, tabs, tm, 10, 0, 73, torch)
    assert rel_l2(got, ref) <= FWD_TOL


def test_noalloc_gather_at_the_sample_limit():
    """M exactly at the 2D limit is served (and matches the oracle)."""
    import torch
    rng = np.random.default_rng(80)
    K, J, L = [128, 128], [6, 6], [1024, 1024]
    tabs = [mb.minmax_kb_table(64, 6, 128, 1024)] * 2
    tm = rng.uniform(-64, 64, (M_MAX_2D, 2))
    got, ref = _oracle_case(2, K, J, L, tabs, tm, 1, 0, 81, torch)
    assert got.shape == (M_MAX_2D, 1)
    assert rel_l2(got, ref) <= FWD_TOL
