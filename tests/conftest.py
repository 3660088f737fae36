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
