"""GPU: density compensation through the C ABI against the FP64 oracle.

mirt_dcf_pipe / mirt_dcf_jackson run the plan's FP32 spread and gather with an
FP64 ratio update; the oracle (oracle/dcf_ref.py) runs the same loop in FP64 on
the reference's table kernels.  Tolerance on the weights: relative L2
<= 2e-4 (about 20 ratio updates, each with an FP32 P P' w); the update counts
must agree exactly and the last residual to 1e-4.
"""
from __future__ import annotations

import numpy as np
import pytest

import mirt_b200 as mb
from mirt_b200 import workloads as wl
from conftest import rel_l2
from oracle import dcf_ref
from oracle import nufft_ref as nr

pytestmark = pytest.mark.gpu

W_TOL = 2e-4


def _plan(om, N, K, moff=None):
    return mb.NufftPlan(om, (N, N), (6, 6), (K, K), n_shift=(N / 2, N / 2), Ld=1024, ncol=1,
                        slice_moff=moff)


def _st(om, N, K):
    return nr.nufft_init_table(om, (N, N), (6, 6), (K, K), (N / 2, N / 2), (1024, 1024))


def test_pipe_single_trajectory():
    om = wl.radial(64, 128)                      # the 64 x 128 radial geometry, K = 128^2
    G = _plan(om, 64, 128)
    w, iters, resid = mb.dcf_pipe(G, niter=20, thresh=0.02, return_info=True)
    ref, it_ref, r_ref = dcf_ref.dcf_pipe(_st(om, 64, 128), niter=20, thresh=0.02)
    assert iters[0] == it_ref
    assert abs(resid[0] - r_ref) <= 1e-4
    assert rel_l2(w.cpu().numpy(), ref) <= W_TOL


def test_pipe_batched_uneven_slices():
    """Three trajectories of uneven length in one plan: each slice iterates
    and stops on its own residual, as three separate reference calls would."""
    rng = np.random.default_rng(4)
    oms = [wl.ga_radial(90, 128), wl.vd_spiral(12, 400, 64, alpha=1.3),
           wl.vd_random(9000, rng)]
    moff = np.concatenate([[0], np.cumsum([len(o) for o in oms])])
    G = _plan(np.concatenate(oms), 64, 128, moff)
    w, iters, resid = mb.dcf_pipe(G, niter=25, thresh=0.05, return_info=True)
    w = w.cpu().numpy()
    for s, om in enumerate(oms):
        ref, it_ref, r_ref = dcf_ref.dcf_pipe(_st(om, 64, 128), niter=25, thresh=0.05)
        assert iters[s] == it_ref, s
        assert abs(resid[s] - r_ref) <= 1e-4, s
        assert rel_l2(w[moff[s]:moff[s + 1]], ref) <= W_TOL, s


def test_pipe_runs_niter_plus_one_updates_without_threshold():
    om = wl.vd_spiral(8, 256, 32)
    G = _plan(om, 32, 64)
    w, iters, _ = mb.dcf_pipe(G, niter=6, thresh=0.0, return_info=True)
    assert iters[0] == 7
    ref, it_ref, _ = dcf_ref.dcf_pipe(_st(om, 32, 64), niter=6, thresh=0.0)
    assert it_ref == 7
    assert rel_l2(w.cpu().numpy(), ref) <= W_TOL


def test_jackson_and_api():
    om = wl.ga_radial(50, 128)
    G = _plan(om, 64, 128)
    w = mb.ir_mri_density_comp(om / (2 * np.pi), "jackson", G=G)
    ref = dcf_ref.dcf_jackson(_st(om, 64, 128))
    assert rel_l2(w, ref) <= 1e-5
    wp = mb.ir_mri_density_comp(om / (2 * np.pi), "pipe", G=G, arg_pipe={"niter": 10, "fov": 2.0})
    refp, _, _ = dcf_ref.dcf_pipe(_st(om, 64, 128), niter=10, fov=2.0)
    assert rel_l2(wp, refp) <= W_TOL


def test_pipe_needs_single_column_plan():
    """The C ABI refuses a multi-column plan (the Python wrapper checks first)."""
    import ctypes as C
    import torch
    from mirt_b200._lib import check
    G = mb.NufftPlan(wl.radial(8, 32), (16, 16), (6, 6), (32, 32), Ld=256, ncol=2)
    w = torch.ones(G.Mtot, dtype=torch.float64, device="cuda")
    with pytest.raises(mb.MirtError, match="single-column"):
        check(G.lib.mirt_dcf_pipe(G.handle, C.c_void_p(w.data_ptr()), 1, 5, 0.02, None, None,
                                  None, None))
