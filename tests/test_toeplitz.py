"""Toeplitz Gram restatement (CPU): the kernel built from two adjoint table
NUFFTs (Gnufft_gram_init2) reproduces the exact DTFT Gram operator to the
table NUFFT's accuracy, its spectrum is real (Hermitian kernel), and the
weighted operator is the weighted Gram."""
import numpy as np
import pytest

from mirt_b200 import workloads as wl
from oracle import toeplitz_ref as tr


@pytest.mark.parametrize("weighted", [False, True])
def test_kernel_gram_matches_exact_dtft(weighted):
    rng = np.random.default_rng(1)
    N, K = (24, 20), (48, 40)
    om = wl.ga_radial(30, 48)
    w = rng.uniform(0.5, 2, len(om)) if weighted else None
    H = tr.gram_kernel(om, N, K, w=w)
    assert np.abs(H.imag).max() <= 1e-12 * np.abs(H).max()
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    a = tr.gram_apply(H, x)
    b = tr.gram_exact(om, N, x, w)
    assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b)
