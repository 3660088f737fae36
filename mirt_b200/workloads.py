"""Seeded synthetic inputs for the benchmark configurations.

No public dataset is involved: every array here is generated from a seed with
the shapes and value distributions the configurations name.

* radial trajectories: uniformly spaced spokes, and golden-angle spokes with
  the angle step pi*(sqrt(5)-1)/2 from pi/2 and readout positions
  (-(Nro/2-1) .. Nro/2)/Nro in cycles/sample (the sampling of
  mri/ir_mri_kspace_ga_radial.m:34-53), scaled to radians
* 3D kooshball: spokes through the centre along directions on a Fibonacci
  sphere
* variable-density spirals and random variable-density point sets (the
  training trajectories of the learned density compensation)
* phantoms: random ellipses / ellipsoids with amplitude U[0,1] and phase
  U[-pi, pi)
* coil maps: smooth complex Gaussian bumps with seeded centres and widths
"""
from __future__ import annotations

import numpy as np

GOLDEN_ANGLE = np.pi * (np.sqrt(5) - 1) / 2


def radial(nspoke: int, nread: int) -> np.ndarray:
    """[nspoke*nread, 2] radians, spokes at angles k*pi/nspoke, readout [-pi, pi)."""
    r = np.linspace(-np.pi, np.pi, nread, endpoint=False)
    ang = np.arange(nspoke) * np.pi / nspoke
    return np.stack([np.outer(np.cos(ang), r).ravel(), np.outer(np.sin(ang), r).ravel()], 1)


def ga_radial(nspoke: int, nro: int, start: float = np.pi / 2) -> np.ndarray:
    """[nro*nspoke, 2] radians, golden-angle spokes, readout fastest."""
    phi = np.arange(nspoke) * GOLDEN_ANGLE + start
    rho = np.arange(-(nro // 2 - 1), nro // 2 + 1) / nro
    kx = np.outer(rho, np.cos(phi))
    ky = np.outer(rho, np.sin(-phi))
    return 2 * np.pi * np.stack([kx.ravel(order="F"), ky.ravel(order="F")], 1)


def vd_spiral(ninterleave: int, nsamp: int, N: int, alpha: float = 1.5) -> np.ndarray:
    """[ninterleave*nsamp, 2] radians: variable-density spiral interleaves.

    Radius pi * t**alpha and angle 2 pi * turns * t for t in [0, 1], with
    turns = N / (2 ninterleave) (Nyquist-spaced turns at the edge for
    alpha = 1); alpha > 1 samples the centre more densely.  Interleave i is
    rotated by 2 pi i / ninterleave; samples of one interleave are contiguous.
    """
    t = np.linspace(0, 1, nsamp)
    turns = N / (2.0 * ninterleave)
    r = np.pi * t ** alpha
    th = 2 * np.pi * turns * t
    rot = 2 * np.pi * np.arange(ninterleave) / ninterleave
    a = th[None, :] + rot[:, None]
    return np.stack([(r * np.cos(a)).ravel(), (r * np.sin(a)).ravel()], 1)


def vd_random(M: int, rng: np.random.Generator, gamma: float = 1.6) -> np.ndarray:
    """[M, 2] radians: random variable-density points, radius pi * u**gamma
    (u ~ U[0, 1]), angle ~ U[0, 2 pi); gamma > 1 concentrates the centre."""
    r = np.pi * rng.uniform(0, 1, M) ** gamma
    a = rng.uniform(0, 2 * np.pi, M)
    return np.stack([r * np.cos(a), r * np.sin(a)], 1)


def kooshball(nspoke: int, nro: int) -> np.ndarray:
    """[nspoke*nro, 3] radians: spokes along Fibonacci-sphere directions."""
    i = np.arange(nspoke) + 0.5
    z = 1 - 2 * i / nspoke
    r = np.sqrt(1 - z * z)
    th = np.pi * (1 + np.sqrt(5)) * i
    dirs = np.stack([r * np.cos(th), r * np.sin(th), z], 1)
    rho = np.arange(-(nro // 2 - 1), nro // 2 + 1) / nro * 2 * np.pi
    return (dirs[:, None, :] * rho[None, :, None]).reshape(-1, 3)


def ellipses(N: int, n: int, rng: np.random.Generator) -> np.ndarray:
    """[N, N] complex image (index [n1, n2]) of n random ellipses."""
    x, y = np.meshgrid(np.linspace(-1, 1, N), np.linspace(-1, 1, N), indexing="ij")
    img = np.zeros((N, N), complex)
    for _ in range(n):
        cx, cy = rng.uniform(-0.5, 0.5, 2)
        rx, ry = rng.uniform(0.05, 0.4, 2)
        th = rng.uniform(0, np.pi)
        a = rng.uniform(0, 1) * np.exp(1j * rng.uniform(-np.pi, np.pi))
        xr = (x - cx) * np.cos(th) + (y - cy) * np.sin(th)
        yr = -(x - cx) * np.sin(th) + (y - cy) * np.cos(th)
        img[(xr / rx) ** 2 + (yr / ry) ** 2 <= 1] += a
    return img


def ellipsoids(N: int, n: int, rng: np.random.Generator) -> np.ndarray:
    """[N, N, N] complex volume of n random ellipsoids."""
    g = np.linspace(-1, 1, N, dtype=np.float32)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    vol = np.zeros((N, N, N), np.complex64)
    for _ in range(n):
        c = rng.uniform(-0.4, 0.4, 3)
        r = rng.uniform(0.05, 0.35, 3)
        a = rng.uniform(0, 1) * np.exp(1j * rng.uniform(-np.pi, np.pi))
        inside = (((x - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2
                  + ((z - c[2]) / r[2]) ** 2) <= 1
        vol[inside] += a
    return vol


def coil_maps(shape, ncoil: int, rng: np.random.Generator) -> np.ndarray:
    """[*shape, ncoil] smooth complex Gaussian-bump sensitivities."""
    axes = [np.linspace(-1, 1, n, dtype=np.float32) for n in shape]
    grids = np.meshgrid(*axes, indexing="ij")
    maps = np.empty(tuple(shape) + (ncoil,), np.complex64)
    for c in range(ncoil):
        ang = 2 * np.pi * c / ncoil
        centre = [1.2 * np.cos(ang), 1.2 * np.sin(ang)] + [rng.uniform(-0.5, 0.5)] * (len(shape) - 2)
        width = rng.uniform(0.6, 1.2)
        d2 = sum((g - c0) ** 2 for g, c0 in zip(grids, centre))
        phase = rng.uniform(-np.pi, np.pi) + 0.5 * grids[0] * rng.uniform(-1, 1)
        maps[..., c] = np.exp(-d2 / (2 * width ** 2)) * np.exp(1j * phase)
    return maps


def batch_ga_radial(nslice: int, spoke_lo: int, spoke_hi: int, nro: int,
                    rng: np.random.Generator):
    """Uneven golden-angle slices: (om [Mtot, 2], slice offsets [nslice+1], spokes)."""
    spokes = rng.integers(spoke_lo, spoke_hi + 1, nslice)
    oms = [ga_radial(int(s), nro, start=np.pi / 2 + rng.uniform(0, np.pi)) for s in spokes]
    moff = np.concatenate([[0], np.cumsum([len(o) for o in oms])]).astype(np.int64)
    return np.concatenate(oms), moff, spokes


def cgsense_problems(nprob: int, rng: np.random.Generator, Ns=(128, 192, 256),
                     coils=(8, 16, 24, 32), R: int = 4, snr_db: float = 30.0):
    """Seeded CG-SENSE problems: image size N ~ U(Ns), coils C ~ U(coils),
    golden-angle radial at undersampling R (readout 2N, ceil(pi N / 2 / R)
    spokes), smooth coil maps, an ellipse phantom; the data and its noise
    level (snr_db) are formed by the caller's forward operator.
    Returns dicts with N, C, om [M, 2], sens [N2, N1, C], xtrue [N2, N1], snr_db."""
    out = []
    for _ in range(nprob):
        N = int(rng.choice(Ns))
        C = int(rng.choice(coils))
        nspoke = int(np.ceil(np.pi * N / 2 / R))
        om = ga_radial(nspoke, 2 * N, start=rng.uniform(0, np.pi))
        sens = coil_maps((N, N), C, rng).transpose(1, 0, 2)
        xt = ellipses(N, 10, rng).T.astype(np.complex64)
        out.append(dict(N=N, C=C, om=om, sens=np.ascontiguousarray(sens), xtrue=xt,
                        snr_db=snr_db))
    return out
