"""GPU parity of the table gather / spread against the oracle.

Tolerances (FP32 arithmetic, FP64 table-index selection): relative L2
<= 1e-6 for the forward gather and <= 1e-5 for the adjoint spread, against the
reference's FP64 kernels (golden vectors, or oracle/_ref built from the
reference sources, or the bit-identical restatement when neither is here).
"""
from __future__ import annotations

import numpy as np
import pytest

import mirt_b200 as mb
import oracle
from conftest import load_golden, ref_impl, rel_l2

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-6
ADJ_TOL = 1e-5


def _i32(v):
    return np.asarray(v, dtype=np.int32)


def _fwd(D, ck, h, J, L, tm, K, order):
    N = ck.shape[1]
    ckr = ck.reshape(tuple(K) + (N,), order="F")
    o = None if order is None else _i32([order])
    if D == 1:
        return mb.interp1_table_mex(ck, h[0], _i32(J), _i32(L), tm, o)
    if D == 2:
        return mb.interp2_table_mex(ckr, h[0], h[1], _i32(J), _i32(L), tm, o)
    if D == 3:
        return mb.interp3_table_mex(ckr, h[0], h[1], h[2], _i32(J), _i32(L), tm, o)
    return mb.interp4_table_mex(ckr, h[0], h[1], h[2], h[3], _i32(J), _i32(L), tm, o)


def _adj(D, fm, h, J, L, tm, K, order):
    o = None if order is None else _i32([order])
    if D == 1:
        return mb.interp1_table_adj_mex(fm, h[0], _i32(J), _i32(L), tm, _i32(K), o)
    if D == 2:
        return mb.interp2_table_adj_mex(fm, h[0], h[1], _i32(J), _i32(L), tm, _i32(K), o)
    if D == 3:
        return mb.interp3_table_adj_mex(fm, h[0], h[1], h[2], _i32(J), _i32(L), tm, _i32(K), o)
    return mb.interp4_table_adj_mex(fm, h[0], h[1], h[2], h[3], _i32(J), _i32(L), tm, _i32(K), o)


@pytest.mark.parametrize("i", range(24))
def test_mex_matches_golden(i):
    c = load_golden()[i]
    D = c["D"]
    fwd = _fwd(D, c["ck"], c["h"], c["J"], c["L"], c["tm"], c["K"], c["order"])
    assert fwd.shape == c["fwd"].shape
    assert rel_l2(fwd, c["fwd"]) <= FWD_TOL
    adj = _adj(D, c["fm"], c["h"], c["J"], c["L"], c["tm"], c["K"], c["order"])
    assert adj.shape == c["adj"].shape
    assert rel_l2(adj, c["adj"]) <= ADJ_TOL


def _radial(nspoke, nread):
    r = np.linspace(-np.pi, np.pi, nread, endpoint=False)
    ang = np.arange(nspoke) * np.pi / nspoke
    return np.stack([np.outer(np.cos(ang), r).ravel(), np.outer(np.sin(ang), r).ravel()], 1)


@pytest.mark.parametrize("case", [0, 1, 2], ids=["1d", "2d", "3d"])
def test_mex_delta_known_answer(case):
    """nufft/interp_table_test.m's inputs (a unit grid value, triangle-based
    complex tables, samples across +-2K) through the drop-ins: the known
    answer read straight from the tables (FP32 tables: within 1e-6), and the
    adjoint of single unit samples."""
    from conftest import delta_known_answer, interp_table_test_cases
    c = interp_table_test_cases()[case]
    K, J, L, h, k0, tm = c["K"], c["J"], c["L"], c["h"], c["k0"], c["tm"]
    D = len(K)
    ck = np.zeros((int(np.prod(K)), 1), dtype=np.complex128)
    kk = np.ravel_multi_index(k0, K, order="F")
    ck[kk, 0] = c["val"]
    ans = c["val"] * delta_known_answer(K, J, L, h, k0, tm)
    fm = _fwd(D, ck, h, J, L, tm, K, None)[:, 0]
    assert np.max(np.abs(fm - ans)) <= 1e-6
    ms = [0, len(tm) // 3, len(tm) - 1]
    e = np.zeros((len(tm), len(ms)), dtype=np.complex128)
    e[ms, range(len(ms))] = 1
    adj = _adj(D, e, h, J, L, tm, K, None)
    for i, m in enumerate(ms):
        want = np.conj(delta_known_answer(K, J, L, h, k0, tm[m:m + 1])[0])
        assert abs(adj[kk, i] - want) <= 1e-6


@pytest.mark.parametrize("N", [1, 3, 8, 32, 40])
def test_minmax_tables_2d_columns(N):
    """C1 geometry (K=128^2, J=6, L=1024, radial 64x128) with N columns,
    exercising every lane width of the kernels."""
    rng = np.random.default_rng(N)
    K, J, L = [128, 128], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(64, 6, 128, 1024)] * 2
    om = _radial(64, 128)
    tm = om / (2 * np.pi / 128)
    ck = rng.standard_normal((128 * 128, N)) + 1j * rng.standard_normal((128 * 128, N))
    fm = rng.standard_normal((len(tm), N)) + 1j * rng.standard_normal((len(tm), N))
    ref_f = oracle.interp_for(ck, h, J, L, tm, K, 0, impl=ref_impl(), nthreads=8)
    ref_a = oracle.interp_adj(fm, h, J, L, tm, K, 0, impl=ref_impl(), nthreads=8)
    assert rel_l2(_fwd(2, ck, h, J, L, tm, K, None), ref_f) <= FWD_TOL
    assert rel_l2(_adj(2, fm, h, J, L, tm, K, None), ref_a) <= ADJ_TOL


@pytest.mark.parametrize("variant", ["cx0", "re0", "re1"])
@pytest.mark.parametrize("D", [1, 2, 3])
def test_random_geometry(D, variant):
    """Non-power-of-two grids, J != 6 (generic kernels), wrap far outside [0, K)."""
    rng = np.random.default_rng(100 + D)
    K = [37, 29, 19][:D]
    J = [5, 7, 4][:D]
    L = [128, 64, 256][:D]
    cx = variant == "cx0"
    order = 1 if variant == "re1" else 0
    h = [np.exp(-np.linspace(-j / 2, j / 2, j * l + 1) ** 2)
         * (np.exp(0.4j * np.linspace(-j / 2, j / 2, j * l + 1)) if cx else 1)
         for j, l in zip(J, L)]
    M = 3000
    tm = rng.uniform(-3 * max(K), 3 * max(K), (M, D))
    tm[:50] = np.round(tm[:50] * 2) / 2
    N = 5
    nk = int(np.prod(K))
    ck = rng.standard_normal((nk, N)) + 1j * rng.standard_normal((nk, N))
    fm = rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N))
    ref_f = oracle.interp_for(ck, h, J, L, tm, K, order, impl=ref_impl())
    ref_a = oracle.interp_adj(fm, h, J, L, tm, K, order, impl=ref_impl())
    assert rel_l2(_fwd(D, ck, h, J, L, tm, K, order), ref_f) <= FWD_TOL
    assert rel_l2(_adj(D, fm, h, J, L, tm, K, order), ref_a) <= ADJ_TOL


@pytest.mark.parametrize("variant", ["cx0", "re0", "re1"])
def test_4d_random_geometry(variant):
    """4D gateways (interp4_table1_for.c / interp4_table1_adj.c) on the 3D
    kernels: generic J, K4 < J4 (a 4th-dimension tap wraps twice),
    coordinates far outside [0, K), several columns."""
    rng = np.random.default_rng(404)
    K = [17, 13, 11, 5]
    J = [5, 6, 4, 6]
    L = [64, 128, 32, 64]
    cx = variant == "cx0"
    order = 1 if variant == "re1" else 0
    h = [np.exp(-np.linspace(-j / 2, j / 2, j * l + 1) ** 2)
         * (np.exp(0.4j * np.linspace(-j / 2, j / 2, j * l + 1)) if cx else 1)
         for j, l in zip(J, L)]
    M, N = 2000, 3
    tm = rng.uniform(-3 * max(K), 3 * max(K), (M, 4))
    tm[:40] = np.round(tm[:40] * 2) / 2
    nk = int(np.prod(K))
    ck = rng.standard_normal((nk, N)) + 1j * rng.standard_normal((nk, N))
    fm = rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N))
    ref_f = oracle.interp_for(ck, h, J, L, tm, K, order, impl=ref_impl())
    ref_a = oracle.interp_adj(fm, h, J, L, tm, K, order, impl=ref_impl())
    assert rel_l2(_fwd(4, ck, h, J, L, tm, K, order), ref_f) <= FWD_TOL
    assert rel_l2(_adj(4, fm, h, J, L, tm, K, order), ref_a) <= ADJ_TOL


def test_4d_plan_multislice_phase_autotuned():
    """4D device plan: uneven slices (one empty), 8 coils, a per-sample phase,
    J = 6 (the 3D plan underneath may pick its line sweep and TMA gather),
    against the oracle per slice before and after autotuning."""
    import torch
    rng = np.random.default_rng(44)
    K, J, L = [24, 20, 18, 9], [6, 6, 6, 6], [256, 256, 256, 256]
    h = [np.exp(-np.linspace(-3, 3, 6 * 256 + 1) ** 2 / 2)
         * np.exp(0.3j * d * np.linspace(-3, 3, 6 * 256 + 1)) for d in range(4)]
    counts = [1500, 0, 900]
    moff = np.concatenate([[0], np.cumsum(counts)])
    tm = np.concatenate([rng.uniform(-30, 30, (c, 4)) for c in counts])
    ph = np.exp(1j * rng.uniform(0, 2 * np.pi, len(tm)))
    C, S = 8, len(counts)
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff, phase=ph)
    assert plan.grid_shape == (S, 9, 18, 20, 24, C)
    ck = rng.standard_normal(plan.grid_shape) + 1j * rng.standard_normal(plan.grid_shape)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    ck_d = torch.from_numpy(ck.astype(np.complex64)).cuda()
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()

    def check():
        out_f = plan.forward(ck_d).cpu().numpy()
        out_a = plan.adjoint(fm_d).cpu().numpy()
        for s in range(S):
            sl = slice(moff[s], moff[s + 1])
            got_a = np.transpose(out_a[s], (3, 2, 1, 0, 4)).reshape(-1, C, order="F")
            if not counts[s]:
                assert not got_a.any()
                continue
            cks = np.transpose(ck[s], (3, 2, 1, 0, 4)).reshape(-1, C, order="F")
            ref_f = oracle.interp_for(cks, h, J, L, tm[sl], K, 0, impl=ref_impl())
            assert rel_l2(out_f[sl], ph[sl, None] * ref_f) <= FWD_TOL
            ref_a = oracle.interp_adj(np.conj(ph[sl, None]) * fm[sl], h, J, L, tm[sl], K, 0,
                                      impl=ref_impl())
            assert rel_l2(got_a, ref_a) <= ADJ_TOL
        return out_a

    before = check()
    plan.autotune()
    after = check()
    assert rel_l2(after, before) <= ADJ_TOL
    plan.close()


def test_3d_minmax_multicolumn():
    """3D J=6 (the fixed-J kernels), several columns (the reference's 3D
    gateway accepts only N = 1; this drop-in lifts that)."""
    rng = np.random.default_rng(5)
    K, J, L = [32, 32, 32], [6, 6, 6], [512, 512, 512]
    h = [mb.minmax_kb_table(16, 6, 32, 512)] * 3
    M = 4000
    om = rng.uniform(-np.pi, np.pi, (M, 3))
    tm = om / (2 * np.pi / 32)
    N = 8
    ck = rng.standard_normal((32 ** 3, N)) + 1j * rng.standard_normal((32 ** 3, N))
    fm = rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N))
    ref_f = oracle.interp_for(ck, h, J, L, tm, K, 0, impl=ref_impl(), nthreads=8)
    ref_a = oracle.interp_adj(fm, h, J, L, tm, K, 0, impl=ref_impl(), nthreads=8)
    assert rel_l2(_fwd(3, ck, h, J, L, tm, K, None), ref_f) <= FWD_TOL
    assert rel_l2(_adj(3, fm, h, J, L, tm, K, None), ref_a) <= ADJ_TOL


def test_adjoint_is_deterministic():
    """The spread has no atomics: two runs agree bit for bit."""
    rng = np.random.default_rng(9)
    K, J, L = [64, 64], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(32, 6, 64, 1024)] * 2
    tm = rng.uniform(-40, 40, (20000, 2))
    fm = rng.standard_normal((20000, 4)) + 1j * rng.standard_normal((20000, 4))
    a = _adj(2, fm, h, J, L, tm, K, None)
    b = _adj(2, fm, h, J, L, tm, K, None)
    assert np.array_equal(a, b)


def test_empty_and_single_sample():
    h = [mb.minmax_kb_table(8, 6, 16, 64)] * 2
    J, L, K = [6, 6], [64, 64], [16, 16]
    ck = np.ones((256, 1), complex)
    out = _fwd(2, ck, h, J, L, np.zeros((0, 2)), K, None)
    assert out.shape == (0, 1)
    adj = _adj(2, np.zeros((0, 1), complex), h, J, L, np.zeros((0, 2)), K, None)
    assert adj.shape == (256, 1) and not adj.any()
    tm = np.array([[3.25, -7.5]])
    ref = oracle.interp_for(ck, h, J, L, tm, K, 0, impl=ref_impl())
    assert rel_l2(_fwd(2, ck, h, J, L, tm, K, None), ref) <= FWD_TOL


def test_plan_multislice_uneven():
    """Device plan over several slices of uneven length (one launch each way)
    against the oracle per slice."""
    import torch
    rng = np.random.default_rng(21)
    K, J, L = [96, 80], [6, 6], [512, 512]
    h = [mb.minmax_kb_table(48, 6, 96, 512), mb.minmax_kb_table(40, 6, 80, 512)]
    counts = [700, 0, 1300, 50, 2000]
    moff = np.concatenate([[0], np.cumsum(counts)])
    tm = np.concatenate([rng.uniform(-60, 60, (c, 2)) for c in counts])
    C = 8
    S = len(counts)
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff)
    ck = (rng.standard_normal((S, 80, 96, C)) + 1j * rng.standard_normal((S, 80, 96, C)))
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    ck_d = torch.from_numpy(ck.astype(np.complex64)).cuda()
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    out_f = plan.forward(ck_d).cpu().numpy()
    out_a = plan.adjoint(fm_d).cpu().numpy()
    for s in range(S):
        sl = slice(moff[s], moff[s + 1])
        cks = np.transpose(ck[s], (1, 0, 2)).reshape(-1, C, order="F")
        ref_f = oracle.interp_for(cks, h, J, L, tm[sl], K, 0, impl=ref_impl())
        if counts[s]:
            assert rel_l2(out_f[sl], ref_f) <= FWD_TOL
        ref_a = oracle.interp_adj(fm[sl], h, J, L, tm[sl], K, 0, impl=ref_impl())
        got_a = np.transpose(out_a[s], (1, 0, 2)).reshape(-1, C, order="F")
        if counts[s]:
            assert rel_l2(got_a, ref_a) <= ADJ_TOL
        else:
            assert not got_a.any()
    plan.close()


@pytest.mark.parametrize("C", [1, 8, 32])
def test_autotuned_plan_keeps_parity(C):
    """Every tile shape the autotuner may pick gives the same (correct) result."""
    import torch
    rng = np.random.default_rng(31 + C)
    K, J, L = [128, 96], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(64, 6, 128, 1024), mb.minmax_kb_table(48, 6, 96, 1024)]
    counts = [3000, 1700]
    moff = np.concatenate([[0], np.cumsum(counts)])
    tm = np.concatenate([rng.uniform(-70, 70, (c, 2)) for c in counts])
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    before = plan.adjoint(fm_d).cpu().numpy()
    cfg = plan.autotune()
    assert cfg["spread_threads"] % 32 == 0
    after = plan.adjoint(fm_d).cpu().numpy()
    for s in range(2):
        sl = slice(moff[s], moff[s + 1])
        ref = oracle.interp_adj(fm[sl], h, J, L, tm[sl], K, 0, impl=ref_impl())
        got = np.transpose(after[s], (1, 0, 2)).reshape(-1, C, order="F")
        assert rel_l2(got, ref) <= ADJ_TOL
    assert rel_l2(after, before) <= ADJ_TOL
    ck = rng.standard_normal(plan.grid_shape) + 1j * rng.standard_normal(plan.grid_shape)
    out = plan.forward(torch.from_numpy(ck.astype(np.complex64)).cuda()).cpu().numpy()
    for s in range(2):
        sl = slice(moff[s], moff[s + 1])
        cks = np.transpose(ck[s], (1, 0, 2)).reshape(-1, C, order="F")
        ref = oracle.interp_for(cks, h, J, L, tm[sl], K, 0, impl=ref_impl())
        assert rel_l2(out[sl], ref) <= FWD_TOL
    plan.close()


@pytest.mark.parametrize("C", [1, 4, 8, 32])
def test_spread_tilings_padded_and_plain(C):
    """Every fixed tiling -- tile shape, warps per tile, spare tile columns
    (bounds-free row update) or none -- gives the oracle's adjoint."""
    import torch
    rng = np.random.default_rng(77 + C)
    K, J, L = [96, 80], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(48, 6, 96, 1024), mb.minmax_kb_table(40, 6, 80, 1024)]
    tm = rng.uniform(-100, 100, (2500, 2))
    tm[:40] = np.round(tm[:40])
    plan = mb.InterpPlan(K, J, L, h, tm, C)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    ref = oracle.interp_adj(fm, h, J, L, tm, K, 0, impl=ref_impl())
    for tile, threads in [((8, 8), 32), ((16, 16), 64), ((32, 8), 32), ((8, 32), 128)]:
        for padc in (0, 5):
            cfg = plan.set_spread(tile, threads, padc)
            assert cfg["spread_padc"] == padc and cfg["spread_tile"][:2] == list(tile)
            got = plan.adjoint(fm_d).cpu().numpy()[0]
            got = np.transpose(got, (1, 0, 2)).reshape(-1, C, order="F")
            assert rel_l2(got, ref) <= ADJ_TOL, (tile, threads, padc)
    plan.close()


def test_spread_tilings_3d_padded():
    import torch
    rng = np.random.default_rng(78)
    K, J, L = [24, 20, 16], [6, 6, 6], [256, 256, 256]
    h = [mb.minmax_kb_table(k // 2, 6, k, 256) for k in K]
    tm = rng.uniform(-40, 40, (1500, 3))
    C = 8
    plan = mb.InterpPlan(K, J, L, h, tm, C)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    ref = oracle.interp_adj(fm, h, J, L, tm, K, 0, impl=ref_impl())
    for tile, threads in [((8, 8, 8), 32), ((16, 8, 8), 64)]:
        for padc in (0, 5):
            plan.set_spread(tile, threads, padc)
            got = plan.adjoint(fm_d).cpu().numpy()[0]
            got = np.transpose(got, (2, 1, 0, 3)).reshape(-1, C, order="F")
            assert rel_l2(got, ref) <= ADJ_TOL, (tile, threads, padc)
    plan.close()


@pytest.mark.parametrize("C", [1, 8, 32])
def test_atomic_spread_matches_oracle(C):
    """Non-deterministic mode: all warps of a tile take whole samples and add
    with shared-memory atomics; the result is the oracle's adjoint to the same
    tolerance, for several tilings, and the autotuner may pick it."""
    import torch
    rng = np.random.default_rng(91 + C)
    K, J, L = [96, 80], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(48, 6, 96, 1024), mb.minmax_kb_table(40, 6, 80, 1024)]
    counts = [2000, 1500]
    moff = np.concatenate([[0], np.cumsum(counts)])
    tm = np.concatenate([rng.uniform(-100, 100, (c, 2)) for c in counts])
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff)
    cfg = plan.set_deterministic(False)
    assert cfg["spread_atomic"] == 1
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    refs = [oracle.interp_adj(fm[moff[s]:moff[s + 1]], h, J, L, tm[moff[s]:moff[s + 1]], K, 0,
                              impl=ref_impl()) for s in range(2)]

    def check():
        out = plan.adjoint(fm_d).cpu().numpy()
        for s in range(2):
            got = np.transpose(out[s], (1, 0, 2)).reshape(-1, C, order="F")
            assert rel_l2(got, refs[s]) <= ADJ_TOL

    check()
    for tile, threads in [((8, 8), 128), ((16, 16), 256), ((32, 8), 256)]:
        plan.set_spread(tile, threads, 0)
        assert plan.config()["spread_atomic"] == 1
        check()
    plan.autotune()
    check()
    plan.close()


def test_atomic_spread_3d():
    import torch
    rng = np.random.default_rng(92)
    K, J, L = [24, 20, 16], [6, 6, 6], [256, 256, 256]
    h = [mb.minmax_kb_table(k // 2, 6, k, 256) for k in K]
    tm = rng.uniform(-40, 40, (1500, 3))
    C = 8
    plan = mb.InterpPlan(K, J, L, h, tm, C)
    plan.set_deterministic(False)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    got = plan.adjoint(torch.from_numpy(fm.astype(np.complex64)).cuda()).cpu().numpy()[0]
    got = np.transpose(got, (2, 1, 0, 3)).reshape(-1, C, order="F")
    ref = oracle.interp_adj(fm, h, J, L, tm, K, 0, impl=ref_impl())
    assert rel_l2(got, ref) <= ADJ_TOL
    plan.close()


@pytest.mark.parametrize("C", [1, 8, 32])
def test_ownership_spread_matches_oracle(C):
    """Ownership spread (2D, J = 6): padded tiles in four colour launches.  A
    dense slice forces split tiles (partial tiles summed by the reduction);
    every tiling gives the oracle's adjoint, bitwise reproducibly."""
    import torch
    rng = np.random.default_rng(71 + C)
    K, J, L = [96, 96], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(48, 6, 96, 1024)] * 2
    tms = [rng.uniform(-60, 60, (1500, 2)), rng.uniform(-3, 3, (5000, 2)),
           rng.uniform(-48, 48, (800, 2))]
    moff = np.concatenate([[0], np.cumsum([len(t) for t in tms])])
    tm = np.concatenate(tms)
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    refs = [oracle.interp_adj(fm[moff[s]:moff[s + 1]], h, J, L, tms[s], K, 0, impl=ref_impl())
            for s in range(3)]
    for tile, threads in [((8, 8), 32), ((16, 8), 64), ((16, 16), 128)]:
        plan.set_spread(tile, threads, 0)
        cfg = plan.set_ownership(True)
        assert cfg["spread_own"] == 1 and cfg["spread_reductions"] > 0
        out = plan.adjoint(fm_d).cpu().numpy()
        for s in range(3):
            got = np.transpose(out[s], (1, 0, 2)).reshape(-1, C, order="F")
            assert rel_l2(got, refs[s]) <= ADJ_TOL, (tile, s)
        assert np.array_equal(out, plan.adjoint(fm_d).cpu().numpy())
    plan.close()


def test_ownership_spread_refused_where_colours_would_overlap():
    K, J, L = [80, 96], [6, 6], [256, 256]
    h = [mb.minmax_kb_table(40, 6, 80, 256), mb.minmax_kb_table(48, 6, 96, 256)]
    tm = np.random.default_rng(0).uniform(-40, 40, (300, 2))
    plan = mb.InterpPlan(K, J, L, h, tm, 4)
    plan.set_spread((16, 16), 32, 0)         # 5 tiles along K1 = 80: odd
    with pytest.raises(mb.MirtError, match="even number of tiles"):
        plan.set_ownership(True)
    plan.close()


@pytest.mark.parametrize("C", [1, 3, 8, 32, 40])
def test_sweep_spread_matches_oracle(C):
    """Row-sweep spread (2D, J = 6): three slices (one dense, one with
    coordinates far outside the grid, wrapping several times), a partial
    coil chunk at C = 3 and 40, bands of 1, 2 and 4 rows, whole rows, uniform
    row segments down to one column (K1 = 96 in 5 segments: a shorter last
    one) and balanced team lists (segments cut at equal visit counts); the oracle's adjoint, bitwise reproducible and
    independent of bands and segments, and the tiled spread's result to FP32
    rounding (another summation order)."""
    import torch
    rng = np.random.default_rng(171 + C)
    K, J, L = [96, 64], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(48, 6, 96, 1024), mb.minmax_kb_table(32, 6, 64, 1024)]
    tms = [rng.uniform(-60, 60, (1500, 2)), rng.uniform(-3, 3, (5000, 2)),
           rng.uniform(-300, 300, (800, 2))]
    moff = np.concatenate([[0], np.cumsum([len(t) for t in tms])])
    tm = np.concatenate(tms)
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    cfg = plan.config()                        # the default for 32-coil chunks: balanced teams
    assert (cfg["spread_sweep"], cfg["spread_sweep_rows"]) == ((-1, 1) if C >= 32 else (0, 1))
    # one-row bands with dense-bin patches (slice 1 is dense): oracle, and the
    # same bits for every segmentation
    plan.set_dense(True)
    dense_first = None
    for nseg in (-1, 1, 5, 96):
        plan.set_sweep(nseg, 1)
        out = plan.adjoint(fm_d).cpu().numpy()
        for s in range(3):
            got = np.transpose(out[s], (1, 0, 2)).reshape(-1, C, order="F")
            assert rel_l2(got, oracle.interp_adj(fm[moff[s]:moff[s + 1]], h, J, L, tms[s], K, 0,
                                                 impl=ref_impl())) <= ADJ_TOL, (nseg, s)
        dense_first = out if dense_first is None else dense_first
        assert np.array_equal(out, dense_first), nseg
    plan.set_dense(False)
    plan.set_sweep(0)
    tiled = plan.adjoint(fm_d).cpu().numpy()
    refs = [oracle.interp_adj(fm[moff[s]:moff[s + 1]], h, J, L, tms[s], K, 0, impl=ref_impl())
            for s in range(3)]
    first = None
    for nseg, rows in [(1, 1), (3, 2), (16, 4), (96, 4), (1, 4), (5, 2), (-1, 1), (-1, 2)]:
        cfg = plan.set_sweep(nseg, rows)
        assert cfg["spread_sweep"] == nseg and cfg["spread_sweep_rows"] == rows
        out = plan.adjoint(fm_d).cpu().numpy()
        for s in range(3):
            got = np.transpose(out[s], (1, 0, 2)).reshape(-1, C, order="F")
            assert rel_l2(got, refs[s]) <= ADJ_TOL, (nseg, rows, s)
        assert np.array_equal(out, plan.adjoint(fm_d).cpu().numpy())
        assert rel_l2(out, tiled) <= 5e-6      # two FP32 summation orders
        if first is None:
            first = out
        assert np.array_equal(out, first)      # neither segments nor bands change the sums
    with pytest.raises(mb.MirtError, match="segments"):
        plan.set_sweep(97)
    with pytest.raises(mb.MirtError, match="rows per band"):
        plan.set_sweep(1, 3)
    plan.set_sweep(False)
    assert np.array_equal(plan.adjoint(fm_d).cpu().numpy(), tiled)
    plan.close()


@pytest.mark.parametrize("order", [0, 1])
def test_sweep_spread_real_tables_phase_small_grid(order):
    """Real tables (order 0 and 1) with a per-sample phase, on grids down to
    K = 6 x 7 where every tap row and column wraps; bands of 2 and 4 rows
    with a partial last band (K2 = 7, 9)."""
    import torch
    rng = np.random.default_rng(5 + order)
    for K in ([6, 7], [12, 9], [40, 24]):
        J, L = [6, 6], [64, 64]
        h = [np.cos(np.linspace(-1.2, 1.2, 6 * 64 + 1)), np.exp(-np.linspace(-2, 2, 6 * 64 + 1) ** 2)]
        tm = rng.uniform(-20, 20, (700, 2))
        ph = np.exp(1j * rng.uniform(-np.pi, np.pi, len(tm)))
        C = 4
        plan = mb.InterpPlan(K, J, L, h, tm, C, order=order, phase=ph)
        plan.set_sweep(1, 4 if K[1] > 7 else 2)
        fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
        got = plan.adjoint(torch.from_numpy(fm.astype(np.complex64)).cuda()).cpu().numpy()[0]
        got = np.transpose(got, (1, 0, 2)).reshape(-1, C, order="F")
        ref = oracle.interp_adj(fm * np.conj(ph)[:, None], h, J, L, tm, K, order, impl=ref_impl())
        assert rel_l2(got, ref) <= ADJ_TOL, K
        plan.close()


@pytest.mark.parametrize("C", [32, 40, 64])
def test_staged_sweep_same_bits(C):
    """The row sweep staged per bin column (mirt_interp_plan_set_staged 1: after
    the ordering pass; 2: reading the caller's samples through the sort
    permutation) gives the unstaged sweep's bits for bands of 1, 2 and 4 rows,
    uniform segments and balanced teams, on three slices (a dense one, one
    wrapping several times) with a per-sample phase, a partial coil chunk at
    C = 40; and the oracle's adjoint.  Dense-bin patches take precedence over
    staging (one-row bands): the same bits as without staging."""
    import torch
    rng = np.random.default_rng(29 + C)
    K, J, L = [96, 64], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(48, 6, 96, 1024), mb.minmax_kb_table(32, 6, 64, 1024)]
    tms = [rng.uniform(-60, 60, (1500, 2)), rng.uniform(-3, 3, (5000, 2)),
           rng.uniform(-300, 300, (800, 2))]
    moff = np.concatenate([[0], np.cumsum([len(t) for t in tms])])
    tm = np.concatenate(tms)
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, len(tm)))
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff, phase=ph)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    refs = [oracle.interp_adj((fm * np.conj(ph)[:, None])[moff[s]:moff[s + 1]], h, J, L, tms[s],
                              K, 0, impl=ref_impl()) for s in range(3)]
    plan.set_dense(False)
    first = None
    for nseg, rows in [(1, 1), (5, 2), (16, 4), (-1, 1), (-1, 4)]:
        plan.set_sweep(nseg, rows)
        plan.set_staged(0)
        base = plan.adjoint(fm_d).cpu().numpy()
        for s in range(3):
            got = np.transpose(base[s], (1, 0, 2)).reshape(-1, C, order="F")
            assert rel_l2(got, refs[s]) <= ADJ_TOL, (nseg, rows, s)
        for mode in (1, 2):
            plan.set_staged(mode)
            assert plan.config()["spread_staged"] == mode
            out = plan.adjoint(fm_d).cpu().numpy()
            assert np.array_equal(out, base), (nseg, rows, mode)
        first = base if first is None else first
        assert np.array_equal(base, first)
    plan.set_dense(True)
    plan.set_sweep(-1, 1)
    plan.set_staged(0)
    dense = plan.adjoint(fm_d).cpu().numpy()
    plan.set_staged(2)
    assert np.array_equal(plan.adjoint(fm_d).cpu().numpy(), dense)
    with pytest.raises(mb.MirtError, match="staged mode"):
        plan.set_staged(3)
    plan.close()
    small = mb.InterpPlan(K, J, L, h, tms[0], 8)
    with pytest.raises(mb.MirtError, match="32-coil"):
        small.set_staged(1)
    small.close()


@pytest.mark.parametrize("order", [0, 1])
def test_staged_sweep_real_tables_phase(order):
    """The staged row sweep with real tables (order 0 and 1) and a per-sample
    phase, 32 coils, grids down to K = 6 x 7 (every tap row and column wraps):
    the unstaged sweep's bits for both staged modes, and the oracle's adjoint."""
    import torch
    rng = np.random.default_rng(41 + order)
    for K in ([6, 7], [40, 24]):
        J, L = [6, 6], [64, 64]
        h = [np.cos(np.linspace(-1.2, 1.2, 6 * 64 + 1)), np.exp(-np.linspace(-2, 2, 6 * 64 + 1) ** 2)]
        tm = rng.uniform(-20, 20, (900, 2))
        ph = np.exp(1j * rng.uniform(-np.pi, np.pi, len(tm)))
        C = 32
        plan = mb.InterpPlan(K, J, L, h, tm, C, order=order, phase=ph)
        plan.set_dense(False)
        rows = 4 if K[1] > 7 else 2
        plan.set_sweep(1, rows)
        plan.set_staged(0)
        fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
        fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
        base = plan.adjoint(fm_d).cpu().numpy()
        for mode in (1, 2):
            plan.set_staged(mode)
            assert np.array_equal(plan.adjoint(fm_d).cpu().numpy(), base), (K, mode)
        got = np.transpose(base[0], (1, 0, 2)).reshape(-1, C, order="F")
        ref = oracle.interp_adj(fm * np.conj(ph)[:, None], h, J, L, tm, K, order, impl=ref_impl())
        assert rel_l2(got, ref) <= ADJ_TOL, K
        plan.close()


def test_sweep_spread_refused_where_it_does_not_apply():
    h = [mb.minmax_kb_table(8, 4, 16, 64)] * 2
    plan = mb.InterpPlan([16, 16], [4, 4], [64, 64], h, np.zeros((10, 2)), 2)
    with pytest.raises(mb.MirtError, match="row-sweep"):
        plan.set_sweep(True)
    plan.close()


@pytest.mark.parametrize("C,K", [(32, (96, 64)), (40, (13, 27)), (64, (40, 33))])
def test_tma_gather_matches_plain_gather_and_oracle(C, K):
    """Gather over TMA-staged tiles and records (2D, J = 6, even C >= 32):
    bitwise the plain gather (same arithmetic and order), the oracle's
    forward to FP32 rounding, coil chunks (C = 40, 64), grids from 13 points
    (where most blocks wrap and read the grid directly), a dense slice (blocks
    split into several work items), coordinates far outside the grid, three
    slices; the plan's fault flag stays clear."""
    import torch
    rng = np.random.default_rng(11 + C)
    J, L = [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(max(K[0] // 2, 6), 6, K[0], 1024),
         mb.minmax_kb_table(max(K[1] // 2, 6), 6, K[1], 1024)]
    tms = [rng.uniform(-40, 40, (2000, 2)), rng.uniform(-3, 3, (3000, 2)),
           rng.uniform(-300, 300, (700, 2))]
    moff = np.concatenate([[0], np.cumsum([len(t) for t in tms])])
    plan = mb.InterpPlan(K, J, L, h, np.concatenate(tms), C, slice_moff=moff)
    assert plan.config()["gather_tma"] == 1      # the default where it applies
    ck = (rng.standard_normal((3, K[1], K[0], C)) + 1j * rng.standard_normal((3, K[1], K[0], C)))
    ckd = torch.from_numpy(ck.astype(np.complex64)).cuda()
    a = plan.forward(ckd).cpu().numpy()
    assert plan.fault() == 0
    assert plan.set_gather(2)["gather_tma"] == 2  # tiles of 16 coils, a half-warp per sample
    assert np.array_equal(plan.forward(ckd).cpu().numpy(), a)
    assert plan.fault() == 0
    plan.set_gather(False)
    b = plan.forward(ckd).cpu().numpy()
    assert np.array_equal(a, b)
    with pytest.raises(mb.MirtError, match="gather mode"):
        plan.set_gather(3)
    for s in range(3):
        ref = oracle.interp_for(np.transpose(ck[s], (1, 0, 2)).reshape(-1, C, order="F"), h, J, L,
                                tms[s], K, 0, impl=ref_impl())
        assert rel_l2(a[moff[s]:moff[s + 1]], ref) <= FWD_TOL, s
    plan.close()


@pytest.mark.parametrize("C,K", [(8, (32, 24, 20)), (10, (12, 9, 16))])
def test_tma_gather_3d_matches_plain_gather_and_oracle(C, K):
    """3D gather over TMA-staged 9 x 9 x 9 tiles of 8 coils (4 x 4 x 4 blocks
    of first taps, items of up to 32 samples): bitwise the plain 3D gather,
    the oracle's forward to FP32 rounding; a partial coil chunk (C = 10), grids
    down to K = 9 (most blocks wrap and read the grid directly), a dense slice
    (blocks split into several items), coordinates far outside the grid, three
    slices; a per-sample phase; the bounded waits' fault path."""
    import torch
    rng = np.random.default_rng(91 + C)
    J, L = [6, 6, 6], [256, 256, 256]
    h = [mb.minmax_kb_table(max(k // 2, 6), 6, k, 256) for k in K]
    tms = [rng.uniform(-20, 20, (1500, 3)), rng.uniform(-2, 2, (3000, 3)),
           rng.uniform(-100, 100, (500, 3))]
    moff = np.concatenate([[0], np.cumsum([len(t) for t in tms])])
    tm = np.concatenate(tms)
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, len(tm)))
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff, phase=ph)
    assert plan.config()["gather_tma"] == 1      # the default where it applies
    ck = (rng.standard_normal((3, K[2], K[1], K[0], C)) +
          1j * rng.standard_normal((3, K[2], K[1], K[0], C)))
    ckd = torch.from_numpy(ck.astype(np.complex64)).cuda()
    a = plan.forward(ckd).cpu().numpy()
    assert plan.fault() == 0
    plan.set_gather(False)
    assert np.array_equal(plan.forward(ckd).cpu().numpy(), a)
    for s in range(3):
        ref = oracle.interp_for(np.transpose(ck[s], (2, 1, 0, 3)).reshape(-1, C, order="F"), h, J,
                                L, tms[s], K, 0, impl=ref_impl()) * ph[moff[s]:moff[s + 1], None]
        assert rel_l2(a[moff[s]:moff[s + 1]], ref) <= FWD_TOL, s
    with pytest.raises(mb.MirtError, match="2D only"):
        plan.set_gather(2)
    plan.set_gather(True)
    plan.set_fault_test(True)                   # no copies: every wait runs out, nothing in flight
    plan.forward(ckd)
    assert plan.fault() == 1
    plan.close()                                # a faulted plan is discarded
    p6 = mb.InterpPlan(K, J, L, h, tms[0], 6)   # C < 8: no 3D TMA blocks
    assert p6.config()["gather_tma"] == 0
    p6.close()


@pytest.mark.parametrize("order", [0, 1])
def test_tma_gather_3d_real_tables(order):
    """3D TMA gather with real tables (order 0 and 1): the plain 3D gather's
    bits and the oracle's forward."""
    import torch
    rng = np.random.default_rng(61 + order)
    K, J, L = [16, 12, 10], [6, 6, 6], [64, 64, 64]
    t = np.linspace(-2, 2, 6 * 64 + 1)
    h = [np.exp(-t ** 2), np.cos(0.6 * t), np.exp(-0.5 * t ** 2)]
    tm = rng.uniform(-12, 12, (2500, 3))
    C = 8
    plan = mb.InterpPlan(K, J, L, h, tm, C, order=order)
    assert plan.config()["gather_tma"] == 1
    ck = rng.standard_normal((1, K[2], K[1], K[0], C)) + 1j * rng.standard_normal((1, K[2], K[1], K[0], C))
    ckd = torch.from_numpy(ck.astype(np.complex64)).cuda()
    a = plan.forward(ckd).cpu().numpy()
    plan.set_gather(False)
    assert np.array_equal(plan.forward(ckd).cpu().numpy(), a)
    ref = oracle.interp_for(np.transpose(ck[0], (2, 1, 0, 3)).reshape(-1, C, order="F"), h, J, L,
                            tm, K, order, impl=ref_impl())
    assert rel_l2(a, ref) <= FWD_TOL
    assert plan.fault() == 0
    plan.close()


def test_tma_gather_real_tables_phase_and_refusal():
    """Real tables, first order, with a per-sample phase: the TMA gather equals
    the plain gather and the oracle; a plan with C = 8 has no TMA blocks."""
    import torch
    rng = np.random.default_rng(3)
    K, J, L = [48, 40], [6, 6], [256, 256]
    h = [np.cos(np.linspace(-1.2, 1.2, 6 * 256 + 1)), np.exp(-np.linspace(-2, 2, 6 * 256 + 1) ** 2)]
    tm = rng.uniform(-30, 30, (4000, 2))
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, len(tm)))
    plan = mb.InterpPlan(K, J, L, h, tm, 32, order=1, phase=ph)
    plan.set_gather(True)
    ck = rng.standard_normal((1, K[1], K[0], 32)) + 1j * rng.standard_normal((1, K[1], K[0], 32))
    ckd = torch.from_numpy(ck.astype(np.complex64)).cuda()
    a = plan.forward(ckd).cpu().numpy()
    plan.set_gather(2)
    assert np.array_equal(a, plan.forward(ckd).cpu().numpy())
    plan.set_gather(False)
    assert np.array_equal(a, plan.forward(ckd).cpu().numpy())
    ref = oracle.interp_for(np.transpose(ck[0], (1, 0, 2)).reshape(-1, 32, order="F"), h, J, L, tm,
                            K, 1, impl=ref_impl()) * ph[:, None]
    assert rel_l2(a, ref) <= FWD_TOL
    assert plan.fault() == 0
    plan.close()
    p8 = mb.InterpPlan(K, J, L, h, tm, 8, order=1)
    assert p8.config()["gather_tma"] == 0
    with pytest.raises(mb.MirtError, match="TMA gather"):
        p8.set_gather(True)
    p8.close()


@pytest.mark.parametrize("C", [8, 16, 32, 40])
def test_3d_line_sweep_matches_oracle(C):
    """3D line sweep (J = 6; warps own 2 x 2, 2 x 1 or single lines for coil
    chunks of 8, 16, 32; C = 40: a partial second chunk): two slices, one dense
    and one wrapping far outside the grid, on a grid of 12 x 10 x 9 points (so
    tap rows and planes wrap); against the oracle, bitwise the same for 1, 2
    and 5 segments and on repeated calls, and the tiled spread to FP32
    rounding."""
    import torch
    rng = np.random.default_rng(300 + C)
    K, J, L = [12, 10, 9], [6, 6, 6], [512, 512, 512]
    h = [mb.minmax_kb_table(k // 2, 6, k, 512) for k in K]
    # slice 0: a cluster of ~100 samples per bin (dense bins, summed into
    # patches before the sweep) around sparse ones
    tms = [np.concatenate([rng.uniform(-1.5, 1.5, (3000, 3)), rng.uniform(-3, 3, (900, 3))]),
           rng.uniform(-60, 60, (700, 3))]
    moff = np.concatenate([[0], np.cumsum([len(t) for t in tms])])
    tm = np.concatenate(tms)
    plan = mb.InterpPlan(K, J, L, h, tm, C, slice_moff=moff)
    fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
    fm_d = torch.from_numpy(fm.astype(np.complex64)).cuda()
    assert plan.config()["spread_sweep"] > 0          # the default for 3D, J = 6
    refs = [oracle.interp_adj(fm[moff[s]:moff[s + 1]], h, J, L, tms[s], K, 0, impl=ref_impl())
            for s in range(2)]
    first = None
    for nseg in (1, 2, 5):
        plan.set_sweep(nseg)
        out = plan.adjoint(fm_d).cpu().numpy()
        for s in range(2):
            got = np.transpose(out[s], (2, 1, 0, 3)).reshape(-1, C, order="F")
            assert rel_l2(got, refs[s]) <= ADJ_TOL, (nseg, s)
        assert np.array_equal(out, plan.adjoint(fm_d).cpu().numpy())
        if first is None:
            first = out
        assert np.array_equal(out, first), nseg
    plan.set_sweep(0)
    tiled = plan.adjoint(fm_d).cpu().numpy()
    assert rel_l2(tiled, first) <= 5e-6
    plan.close()


@pytest.mark.parametrize("order", [0, 1])
def test_3d_line_sweep_real_tables_phase(order):
    """3D line sweep with real tables (order 0 and 1) and a per-sample phase,
    8 coils, on the smallest grids it takes (6 x 7 x 6)."""
    import torch
    rng = np.random.default_rng(310 + order)
    for K in ([6, 7, 6], [16, 12, 20]):
        J, L = [6, 6, 6], [64, 64, 64]
        h = [np.cos(np.linspace(-1.2, 1.2, 6 * 64 + 1)),
             np.exp(-np.linspace(-2, 2, 6 * 64 + 1) ** 2),
             np.cos(np.linspace(-0.9, 0.9, 6 * 64 + 1))]
        tm = np.concatenate([rng.uniform(-20, 20, (900, 3)), rng.uniform(2, 3, (500, 3))])
        ph = np.exp(1j * rng.uniform(-np.pi, np.pi, len(tm)))
        C = 8
        plan = mb.InterpPlan(K, J, L, h, tm, C, order=order, phase=ph)
        plan.set_sweep(3)
        fm = rng.standard_normal((len(tm), C)) + 1j * rng.standard_normal((len(tm), C))
        got = plan.adjoint(torch.from_numpy(fm.astype(np.complex64)).cuda()).cpu().numpy()[0]
        got = np.transpose(got, (2, 1, 0, 3)).reshape(-1, C, order="F")
        ref = oracle.interp_adj(fm * np.conj(ph)[:, None], h, J, L, tm, K, order, impl=ref_impl())
        assert rel_l2(got, ref) <= ADJ_TOL, K
        plan.close()


def test_tma_gather_bounded_wait_fault_path():
    """The TMA gather's bounded waits, made to run out without a GPU fault:
    the test hook arms every stage's barrier for bytes that no copy delivers
    and issues no copy, so each wait ends at its limit with nothing in flight.
    The launch returns, the plan's fault flag reads 1 (and is cleared by the
    read), and the device keeps working: a new plan's gather of the same
    problem matches the oracle."""
    import torch
    rng = np.random.default_rng(404)
    K, J, L = [96, 64], [6, 6], [1024, 1024]
    h = [mb.minmax_kb_table(48, 6, 96, 1024), mb.minmax_kb_table(32, 6, 64, 1024)]
    tm = rng.uniform(-40, 40, (6000, 2))
    C = 32
    ck = rng.standard_normal((96 * 64, C)) + 1j * rng.standard_normal((96 * 64, C))
    ck_d = torch.from_numpy(ck.reshape(64, 96, C).astype(np.complex64)).cuda()[None]
    for mode in (1, 2):                         # tiles of 32 and of 16 coils
        plan = mb.InterpPlan(K, J, L, h, tm, C)
        plan.set_gather(mode)
        plan.set_fault_test(True)
        plan.forward(ck_d)
        assert plan.fault() == 1
        assert plan.fault() == 0
        plan.close()                            # a faulted plan is discarded
    plan = mb.InterpPlan(K, J, L, h, tm, C)
    got = plan.forward(ck_d).cpu().numpy()
    assert plan.fault() == 0
    ref = oracle.interp_for(ck, h, J, L, tm, K, 0, impl=ref_impl(), nthreads=8)
    assert rel_l2(got, ref) <= FWD_TOL
    plan.close()
