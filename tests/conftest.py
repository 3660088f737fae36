"""Shared test set-up.

Markers: ``gpu`` tests need a CUDA device (run with ``-m gpu``); everything
else runs on the CPU.  The session builds the oracle libraries (cheap) and
makes sure libmirt_b200.so exists (built once by ``python -m mirt_b200.build``).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import oracle
    from mirt_b200 import _lib
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        oracle.build()
    if not os.path.exists(_lib.LIB_PATH):
        from mirt_b200 import build
        build.build()
    yield


def ref_impl() -> str:
    """The reference kernels when built here, else the restatement."""
    import oracle
    return "ref" if oracle.ref_available() else "port"


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def load_golden():
    path = os.path.join(ROOT, "tests", "golden", "interp_golden.npz")
    z = np.load(path)
    cases = []
    for i in range(int(z["ncases"])):
        c = {k: z[f"c{i}_{k}"] for k in ("D", "K", "J", "L", "order", "cx", "tm", "ck", "fm",
                                         "fwd", "adj")}
        D = int(c["D"])
        c["h"] = [z[f"c{i}_h{d}"] for d in range(D)]
        c["D"] = D
        c["order"] = int(c["order"])
        c["cx"] = bool(c["cx"])
        cases.append(c)
    return cases


def delta_known_answer(K, J, L, h, k0, tm):
    """Known answer of the table interpolation of a unit grid value at k0 (the
    inputs of nufft/interp_table_test.m): with J <= K per dimension, a sample
    at t sees k0 through at most one tap k = koff + j with k = k0 (mod K), and
    its value is the product over dimensions of the table entries
    h[floor(J L / 2) + floor((t - k) L + 1/2)] (nufft/table/def,table2.h),
    or 0 where no tap reaches k0."""
    tm = np.atleast_2d(np.asarray(tm, dtype=np.float64))
    out = np.ones(tm.shape[0], dtype=np.complex128)
    for d in range(len(K)):
        t = tm[:, d]
        koff = 1 + np.floor(t - J[d] / 2)
        val = np.zeros(len(t), dtype=np.complex128)
        for j in range(J[d]):
            k = koff + j
            hit = np.mod(k, K[d]) == k0[d]
            n = int(np.floor(J[d] * L[d] / 2)) + np.floor((t - k) * L[d] + 0.5).astype(np.int64)
            val[hit] = h[d][n[hit]]
        out *= val
    return out


def interp_table_test_cases():
    """The set-ups of nufft/interp_table_test.m: tables (1 - |t|/(J/2)) and
    i (1 - |t|/(J/2))^2 mixes, one unit grid value, samples across +-2K."""
    hr = lambda t, J: (1 - np.abs(t / (J / 2))) * (np.abs(t) <= J / 2)
    hi = lambda t, J: (1 - np.abs(t / (J / 2))) ** 2 * (np.abs(t) <= J / 2)

    def tabs(J, L, wr, wi):
        return [wr * hr(np.arange(-j / 2 * l, j / 2 * l + 1) / l, j)
                + 1j * wi * hi(np.arange(-j / 2 * l, j / 2 * l + 1) / l, j) for j, l in zip(J, L)]
    c1 = dict(K=[20], J=[6], L=[10], h=tabs([6], [10], 1, 1), k0=[2], val=1.0,
              tm=np.linspace(-40, 40, 2001)[:, None])
    t1, t2 = np.linspace(0, 8, 201), np.linspace(0, 12, 199)
    tt1, tt2 = np.meshgrid(t1, t2, indexing="ij")
    c2 = dict(K=[8, 12], J=[6, 4], L=[32, 16], h=tabs([6, 4], [32, 16], 0, 1), k0=[0, 0], val=-1j,
              tm=np.stack([tt1.ravel(order="F"), tt2.ravel(order="F")], 1))
    t1, t2, t3 = np.linspace(-16, 16, 69), np.linspace(-24, 24, 89), np.array([-1.0, 0.0, 1.0])
    g = np.meshgrid(t1, t2, t3, indexing="ij")
    c3 = dict(K=[8, 12, 4], J=[5, 3, 4], L=[32, 16, 64], h=tabs([5, 3, 4], [32, 16, 64], 1, 0),
              k0=[0, 0, 0], val=1j, tm=np.stack([a.ravel(order="F") for a in g], 1))
    return [c1, c2, c3]
