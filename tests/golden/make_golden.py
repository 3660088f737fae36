"""Generate tests/golden/interp_golden.npz from the reference's own kernels.

    make -C oracle && python tests/golden/make_golden.py

Inputs are seeded and small; outputs come from nufft/table/interp*_table1_*.c
compiled unmodified into oracle/_ref/libmirt_ref.so (oracle/Makefile), run
with the gateways' column loop.  The fixtures pin the oracle restatement and
the GPU kernels on machines where the reference sources are absent.

Cases cover D = 1, 2, 3, 4; complex order-0, real order-0 and real order-1
tables; several columns; unequal J and L per dimension; J = K, and K4 < J4
(a 4th-dimension tap wrapping twice); coordinates that are
integers, half-integers, tiny negatives and far outside [0, K) (periodic wrap).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def cases():
    rng = np.random.default_rng(20240501)
    out = []
    specs = [
        (1, [24], [6], [64], 2),
        (1, [17], [5], [32], 1),
        (2, [16, 12], [6, 6], [64, 32], 3),
        (2, [20, 18], [5, 4], [16, 64], 1),
        (3, [10, 12, 8], [6, 6, 6], [32, 16, 16], 2),
        (3, [9, 8, 11], [4, 5, 3], [8, 16, 32], 1),
        (4, [7, 6, 8, 5], [4, 3, 5, 4], [16, 8, 32, 16], 2),
        (4, [6, 6, 6, 3], [6, 6, 6, 4], [8, 8, 8, 8], 1),
    ]
    for D, K, J, L, N in specs:
        for variant in ("cx0", "re0", "re1"):
            cx = variant == "cx0"
            order = 1 if variant == "re1" else 0
            h = []
            for j, l in zip(J, L):
                n = j * l + 1
                t = np.linspace(-j / 2, j / 2, n)
                base = np.exp(-t ** 2) * (1 + 0.1 * rng.standard_normal(n))
                h.append(base * np.exp(1j * 0.3 * t) if cx else base)
            M = 150
            tm = rng.uniform(-2.5 * max(K), 2.5 * max(K), (M, D))
            tm[:6] = np.round(tm[:6])
            tm[6:10] = np.round(tm[6:10]) + 0.5
            tm[10:12] = 0.0
            tm[12] = -1e-17
            tm[13] = 1e-300
            nk = int(np.prod(K))
            ck = rng.standard_normal((nk, N)) + 1j * rng.standard_normal((nk, N))
            fm = rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N))
            fwd = oracle.interp_for(ck, h, J, L, tm, K, order, impl="ref")
            adj = oracle.interp_adj(fm, h, J, L, tm, K, order, impl="ref")
            out.append(dict(D=D, K=np.array(K), J=np.array(J), L=np.array(L), order=order,
                            cx=cx, h=h, tm=tm, ck=ck, fm=fm, fwd=fwd, adj=adj))
    return out


def main():
    if not oracle.ref_available():
        oracle.build()
    cs = cases()
    flat = {}
    for i, c in enumerate(cs):
        for k, v in c.items():
            if k == "h":
                for d, hd in enumerate(v):
                    flat[f"c{i}_h{d}"] = hd
            else:
                flat[f"c{i}_{k}"] = np.asarray(v)
    flat["ncases"] = np.array(len(cs))
    path = os.path.join(HERE, "interp_golden.npz")
    np.savez_compressed(path, **flat)
    print(path, os.path.getsize(path), "bytes,", len(cs), "cases")


if __name__ == "__main__":
    main()
