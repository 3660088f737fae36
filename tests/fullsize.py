"""Full-size benchmark configurations and their accuracy against the exact DTFT.

Shared by tests/test_gpu_fullsize.py (bounds) and run as a script on a GPU
host to print the per-configuration accuracy table:

    python tests/fullsize.py

Configurations (seeded synthetic inputs, the shapes of the benchmark):

* c1: 64 x 64 image of 10 ellipses, K = 128^2, J = 6, L = 1024, 64 uniformly
  spaced radial spokes x 128 samples; every sample.
* c2: the 256 x 256 ellipse phantom x coil map 0 of slice 0 of the batched
  2D workload (K = 512^2, J = 6, L = 1024, golden-angle spokes x 512); a
  seeded 4,096-sample subset of that slice's trajectory.
* c3: the 128^3 phantom of 20 ellipsoids x coil map 0 (K = 256^3, J = 6,
  L = 512, kooshball 16,384 spokes x 256); a seeded 4,096-sample subset.

For each: relative L2 error of the GPU NUFFT forward / adjoint against the
exact DTFT (nufft/dtft.m:80-112, nufft/dtft_adj.m:40-60), beside the error of
the FP64 oracle (the reference's own kernels with the FP64 glue) against the
same DTFT, which is the table's quantisation floor (the check of
nufft/nufft.m:63-68), and the GPU against that oracle.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

NSUB = 4096

# the batched workloads of bench.py (same seeds): trajectory seed 1234, images seed 99
C2 = dict(D=2, N=256, K=512, J=6, L=1024, ncoil=32, nslice=64, spokes=(100, 400), nro=512)
C3 = dict(D=3, N=128, K=256, J=6, L=512, ncoil=8, nslice=1, spokes=(16384, 16384), nro=256)


def c2_trajectory():
    from mirt_b200 import workloads as wl
    rng = np.random.default_rng(1234)
    om, moff, spokes = wl.batch_ga_radial(C2["nslice"], C2["spokes"][0], C2["spokes"][1],
                                          C2["nro"], rng)
    return om, moff, spokes


def c3_trajectory():
    from mirt_b200 import workloads as wl
    return wl.kooshball(C3["spokes"][0], C3["nro"])


def c2_image_slice0_coil0():
    """[n1, n2] complex128: slice 0's phantom times coil map 0 (bench.make_images order)."""
    from mirt_b200 import workloads as wl
    rng = np.random.default_rng(99)
    N, C = C2["N"], C2["ncoil"]
    maps = wl.coil_maps((N, N), C, rng)
    ph = wl.ellipses(N, 10, rng).astype(np.complex64)
    return (ph * maps[:, :, 0]).astype(np.complex128)


def c3_image_coil0():
    from mirt_b200 import workloads as wl
    rng = np.random.default_rng(99)
    N, C = C3["N"], C3["ncoil"]
    maps = wl.coil_maps((N, N, N), C, rng)
    vol = wl.ellipsoids(N, 20, rng)
    return (vol * maps[..., 0]).astype(np.complex128)


def c1_case():
    from mirt_b200 import workloads as wl
    rng = np.random.default_rng(0)
    om = wl.radial(64, 128)
    x = wl.ellipses(64, 10, rng)
    return dict(om=om, x=x, N=(64, 64), K=(128, 128), J=(6, 6), L=1024, ns=(32, 32))


def c2_case():
    om, moff, _ = c2_trajectory()
    om0 = om[moff[0]:moff[1]]
    idx = np.sort(np.random.default_rng(7).choice(len(om0), NSUB, replace=False))
    N = C2["N"]
    return dict(om=om0[idx], x=c2_image_slice0_coil0(), N=(N, N), K=(C2["K"],) * 2,
                J=(6, 6), L=C2["L"], ns=(N / 2, N / 2))


def c3_case():
    om = c3_trajectory()
    idx = np.sort(np.random.default_rng(8).choice(len(om), NSUB, replace=False))
    N = C3["N"]
    return dict(om=om[idx], x=c3_image_coil0(), N=(N,) * 3, K=(C3["K"],) * 3, J=(6, 6, 6),
                L=C3["L"], ns=(N / 2,) * 3)


CASES = {"c1": c1_case, "c2": c2_case, "c3": c3_case}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def dtft_accuracy(name):
    """Errors of one configuration: GPU and FP64 oracle against the exact DTFT
    (forward and adjoint), and the GPU against the oracle."""
    import mirt_b200 as mb
    import oracle
    from oracle import nufft_ref as nr
    c = CASES[name]()
    om, x, N, K, J, L, ns = c["om"], c["x"], c["N"], c["K"], c["J"], c["L"], c["ns"]
    impl = "ref" if oracle.ref_available() else "port"
    st_o = nr.nufft_init_table(om, N, J, K, ns, L)
    fw = lambda Xk, s: oracle.interp_for(Xk, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                         impl=impl)[:, 0]
    ad = lambda X, s: oracle.interp_adj(X, s["h"], s["Jd"], s["Ld"], s["tm"], s["Kd"], 0,
                                        impl=impl)[:, 0]
    st = mb.nufft_init(om, N, J, K, ns, "table", L, "minmax:kb")
    X = mb.nufft(x, st)
    X_o = nr.nufft(x, st_o, fw)
    X_e = nr.dtft(x, om, ns)
    y = np.random.default_rng(11).standard_normal((len(om), 2)) @ np.array([1, 1j])
    xa = mb.nufft_adj(y, st)
    xa_o = nr.nufft_adj(y, st_o, ad)
    xa_e = nr.dtft_adj(y, om, N, ns)
    st.close()
    return dict(config=name, M=len(om), fwd_gpu_dtft=rel(X, X_e), fwd_oracle_dtft=rel(X_o, X_e),
                adj_gpu_dtft=rel(xa, xa_e), adj_oracle_dtft=rel(xa_o, xa_e),
                fwd_gpu_oracle=rel(X, X_o), adj_gpu_oracle=rel(xa, xa_o), oracle=impl)


def main():
    rows = [dtft_accuracy(n) for n in ("c1", "c2", "c3")]
    print("| config | samples | forward: GPU vs DTFT | forward: FP64 oracle vs DTFT | "
          "adjoint: GPU vs DTFT | adjoint: FP64 oracle vs DTFT | GPU vs oracle (fwd / adj) |")
    print("|---|---|---|---|---|---|---|")
    for r in rows:
        print(f"| {r['config']} | {r['M']} | {r['fwd_gpu_dtft']:.3e} | {r['fwd_oracle_dtft']:.3e} | "
              f"{r['adj_gpu_dtft']:.3e} | {r['adj_oracle_dtft']:.3e} | "
              f"{r['fwd_gpu_oracle']:.2e} / {r['adj_gpu_oracle']:.2e} |")
    print(f"(oracle kernels: {rows[0]['oracle']})")


if __name__ == "__main__":
    main()
