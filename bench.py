#!/usr/bin/env python
"""Benchmark: batched table NUFFT forward + adjoint on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c2s|c1|c3]
    python bench.py --impl reference ...

One step = the forward NUFFT (deapodise + zero-pad, oversampled FFT, table
gather) and the adjoint NUFFT (table spread, inverse FFT, crop + deapodise)
of one batch of slices x coils.  Unit: Msamples/s = sample-coil pairs
processed (forward + adjoint) per second, over all ranks.  Inputs are
resident in HBM for `value`; `e2e` times the same step through the host-buffer
C ABI (mirt_nufft_forward_host / _adjoint_host) with the copies inside.

Default workload (c2): 64 slices, golden-angle radial with U{100..400} spokes
x 512 samples, 32 coils, N = 256^2, K = 512^2, J = 6, L = 1024, all slices in
one launch per kernel.  Data are seeded synthetic ellipse phantoms times
Gaussian-bump coil maps.  Inputs exceed L2 (126 MB), so L2 is not flushed.

--impl reference times the reference's own CPU path on the host cores: the
table kernels nufft/table/interp2_table1_{for,adj}.c (oracle/_ref, built from
the reference sources) with one coil column per thread, scipy.fft for the
oversampled FFT and numpy for the deapodisation, on a bounded sample of the
same workload.

Multi-GPU (torchrun): each rank runs its own batch (weak scaling, no
collective in the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NUFFT fwd+adj Msamples/s & %HBM peak; CG-SENSE s to NRMSE 1e-3, learned vs plain"
UNIT = "Msamples/s"

WORKLOADS = {
    "c2": dict(D=2, N=256, K=512, J=6, L=1024, ncoil=32, nslice=64, spokes=(100, 400), nro=512),
    "c2s": dict(D=2, N=256, K=512, J=6, L=1024, ncoil=32, nslice=4, spokes=(100, 400), nro=512),
    "c2m": dict(D=2, N=256, K=512, J=6, L=1024, ncoil=32, nslice=16, spokes=(100, 400), nro=512),
    "c1": dict(D=2, N=64, K=128, J=6, L=1024, ncoil=1, nslice=1, spokes=(64, 64), nro=128),
    "c3": dict(D=3, N=128, K=256, J=6, L=512, ncoil=8, nslice=1, spokes=(16384, 16384), nro=256),
    "c3s": dict(D=3, N=128, K=256, J=6, L=512, ncoil=8, nslice=1, spokes=(2048, 2048), nro=256),
}


def describe(name, w):
    if w["D"] == 2:
        sp = (f"{w['spokes'][0]}" if w["spokes"][0] == w["spokes"][1]
              else f"U{{{w['spokes'][0]}..{w['spokes'][1]}}}")
        return (f"batched 2D multicoil table NUFFT fwd+adj: {w['nslice']} slices x {sp} "
                f"golden-angle spokes x {w['nro']}, {w['ncoil']} coils, N={w['N']}^2, "
                f"K={w['K']}^2, J={w['J']}, L={w['L']}")
    return (f"3D table NUFFT fwd+adj: kooshball {w['spokes'][0]} spokes x {w['nro']}, "
            f"{w['ncoil']} coils, N={w['N']}^3, K={w['K']}^3, J={w['J']}, L={w['L']}")


def make_trajectory(w, rng):
    from mirt_b200 import workloads as wl
    if w["D"] == 2:
        om, moff, _ = wl.batch_ga_radial(w["nslice"], w["spokes"][0], w["spokes"][1], w["nro"], rng)
        return om, moff
    om = wl.kooshball(w["spokes"][0], w["nro"])
    return om, np.array([0, len(om)], np.int64)


def make_images(w, rng, nslice=None):
    """complex64 [nslice, N.., ncoil] in device layout: phantom x coil maps."""
    from mirt_b200 import workloads as wl
    S = w["nslice"] if nslice is None else nslice
    N, C = w["N"], w["ncoil"]
    if w["D"] == 2:
        maps = wl.coil_maps((N, N), C, rng)                       # [n1, n2, c]
        out = np.empty((S, N, N, C), np.complex64)                # [s, n2, n1, c]
        for s in range(S):
            ph = wl.ellipses(N, 10, rng).astype(np.complex64)      # [n1, n2]
            out[s] = np.transpose(ph[:, :, None] * maps, (1, 0, 2))
        return out
    maps = wl.coil_maps((N, N, N), C, rng)
    vol = wl.ellipsoids(N, 20, rng)
    return np.transpose(vol[..., None] * maps, (2, 1, 0, 3))[None].copy()


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def physical_gpu_index(dev):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if dev < len(ids) and ids[dev].isdigit():
            return int(ids[dev])
    return dev


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_from_profiles(workload, kernel):
    """(DRAM bytes of one call, where they come from) for the dominant kernel
    configuration, looked up in profiles/traffic.json (ncu captures, stated
    there); (None, None) when that configuration was not captured."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        e = t.get(workload, {}).get(kernel)
        if e:
            return e["bytes"], "profiles/traffic.json: " + e["source"]
    except (OSError, ValueError, KeyError):
        pass
    return None, None


# ---------------------------------------------------------------------------
# CPU path of the reference (oracle/_ref kernels + scipy FFT + numpy glue)
# ---------------------------------------------------------------------------
class CpuReference:
    def __init__(self, w, om, moff, n_shift, threads=None):
        import oracle
        from oracle import nufft_ref as nr
        self.oracle = oracle
        self.impl = "ref" if oracle.ref_available() else "port"
        self.kind = "reference" if self.impl == "ref" else "port"
        self.w = w
        D = w["D"]
        self.Nd = (w["N"],) * D
        self.Kd = (w["K"],) * D
        self.Jd = (w["J"],) * D
        self.Ld = (w["L"],) * D
        self.h = [nr.table_1d(w["N"], w["J"], w["K"], w["L"])] * D
        self.sn = nr.scaling_factors(self.Nd, self.Jd, self.Kd)
        self.om, self.moff, self.n_shift = om, moff, np.asarray(n_shift, float)
        allc = oracle.ref_max_threads() if self.impl == "ref" else 1
        # the reference's own behaviour is one core (no threads in nufft/table/);
        # threads > 1 runs one coil column per thread
        self.threads = allc if threads is None else max(1, min(int(threads), allc))

    def step(self, s, x):
        """forward + adjoint of slice s; x [N.., C] (MATLAB order; C columns are
        timed, any number of the workload's coils).  Returns #sample-coils."""
        import scipy.fft as sf
        om = self.om[self.moff[s]:self.moff[s + 1]]
        tm = np.stack([om[:, d] / (2 * np.pi / self.Kd[d]) for d in range(len(self.Kd))], 1)
        ph = np.exp(1j * (om @ self.n_shift))
        C = x.shape[-1]
        D = len(self.Kd)
        ax = tuple(range(D))
        xs = x * self.sn[..., None]
        Xk = sf.fftn(xs, s=self.Kd, axes=ax, workers=self.threads)
        ck = Xk.reshape(-1, C, order="F")
        if self.impl == "ref":
            X = self.oracle.interp_for(ck, self.h, self.Jd, self.Ld, tm, self.Kd, 0,
                                       impl="ref", nthreads=self.threads)
        else:
            X = self.oracle.interp_for(ck, self.h, self.Jd, self.Ld, tm, self.Kd, 0, impl="port")
        X = X * ph[:, None]
        Y = X * np.conj(ph)[:, None]
        if self.impl == "ref":
            ck2 = self.oracle.interp_adj(Y, self.h, self.Jd, self.Ld, tm, self.Kd, 0,
                                         impl="ref", nthreads=self.threads)
        else:
            ck2 = self.oracle.interp_adj(Y, self.h, self.Jd, self.Ld, tm, self.Kd, 0, impl="port")
        g = sf.ifftn(ck2.reshape(self.Kd + (C,), order="F"), axes=ax, norm="forward",
                     workers=self.threads)
        xa = g[tuple(slice(0, n) for n in self.Nd)] * np.conj(self.sn)[..., None]
        assert np.isfinite(xa).all()
        return 2 * len(om) * C

    def timed_sample(self, images, target_s=12.0, max_slices=None, coils=None):
        """Time slices (their first `coils` coils, all if None) until ~target_s of
        CPU work; returns (Msamples/s, slices, sample-coils, seconds)."""
        S = len(self.moff) - 1
        limit = S if max_slices is None else min(S, max_slices)
        units, t0, n = 0, time.perf_counter(), 0
        while n < limit:
            x = self._image(images, n)
            if coils is not None:
                x = x[..., :coils]
            units += self.step(n, x)
            n += 1
            if time.perf_counter() - t0 >= target_s:
                break
        t = time.perf_counter() - t0
        return units / t / 1e6, n, units, t

    def _image(self, images, s):
        D = len(self.Kd)
        axes = tuple(range(D - 1, -1, -1)) + (D,)
        return np.transpose(images[s % len(images)], axes).astype(np.complex128)


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    rng = np.random.default_rng(1234)
    om, moff = make_trajectory(w, rng)
    images = make_images(w, np.random.default_rng(99), nslice=min(4, w["nslice"]))
    n_shift = [w["N"] / 2] * w["D"]
    ref = CpuReference(w, om, moff, n_shift)
    S = len(moff) - 1
    for i in range(args.warmup):
        ref.step(i % S, ref._image(images, i))
    times, units = [], 0
    for i in range(args.steps):
        s = (args.warmup + i) % S
        t0 = time.perf_counter()
        u = ref.step(s, ref._image(images, s))
        times.append(time.perf_counter() - t0)
        units += u
    total = sum(times)
    value = units / total / 1e6
    sample = (f"per step one slice (forward + adjoint, {w['ncoil']} coils) of the workload; "
              f"{args.steps} steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": describe(args.workload, w)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU path
# ---------------------------------------------------------------------------
def combine_over_ranks(t_local, units_local, world, dev):
    """Whole-job (time, units): the slowest rank's time (every rank's batch is
    independent, so the job ends when the last rank does) and the units all
    ranks processed.  One all-reduce each, outside the timed region."""
    if world <= 1:
        return t_local, units_local
    import torch
    import torch.distributed as dist
    tt = torch.tensor([t_local], device=dev, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    uu = torch.tensor([units_local], device=dev, dtype=torch.float64)
    dist.all_reduce(uu, op=dist.ReduceOp.SUM)
    return float(tt.item()), float(uu.item())


def rank_batch(w, rank):
    """The independent batch of slices of one rank (weak scaling): its own
    seeded trajectories; no sample is shared between ranks."""
    rng = np.random.default_rng(1234 + rank)
    return make_trajectory(w, rng)


def run_gpu(args, w):
    import torch
    import torch.distributed as dist

    import mirt_b200 as mb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    om, moff = rank_batch(w, rank)
    Mtot = len(om)
    C = w["ncoil"]
    D = w["D"]
    n_shift = [w["N"] / 2] * D
    plan = mb.NufftPlan(om, (w["N"],) * D, (w["J"],) * D, (w["K"],) * D, n_shift=n_shift,
                        Ld=w["L"], ncol=C, slice_moff=moff)
    t0 = time.perf_counter()
    if args.nondeterministic:
        plan.set_deterministic(False)
    tuned = plan.autotune() if not args.no_autotune else plan.config()
    if args.spread == "sweep" and tuned.get("spread_sweep", 0) == 0:
        tuned = plan.set_sweep(-1, 1)        # the plan's default: balanced teams of one row
    elif args.spread == "tiled" and tuned.get("spread_sweep", 0) != 0:
        tuned = plan.set_sweep(0)
    if args.sweep_config:                       # a fixed row sweep (for captures of one config)
        v = [int(x) for x in args.sweep_config.split(",")]
        tuned = plan.set_sweep(v[0], v[1])
        if len(v) > 3:
            plan.set_dense(bool(v[3]))
        if len(v) > 2:
            plan.set_staged(v[2])
        tuned = plan.config()
    if args.gather_tma is not None:             # a fixed gather (for captures of one form)
        tuned = plan.set_gather(args.gather_tma)
    t_tune = time.perf_counter() - t0
    img_np = make_images(w, np.random.default_rng(99 + rank))
    if img_np.shape[0] != plan.nslice:
        reps = -(-plan.nslice // img_np.shape[0])
        img_np = np.concatenate([img_np] * reps)[:plan.nslice]
    x = torch.from_numpy(img_np).to(dev)
    X = torch.empty(plan.sample_shape, dtype=torch.complex64, device=dev)
    xa = torch.empty(plan.image_shape, dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        plan.forward(x, out=X)
        plan.adjoint(X, out=xa)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # eager steps, timed for reference (outside the contract's timed region)
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    for _ in range(args.steps):
        step()
    eb.record(stream)
    torch.cuda.synchronize()
    eager_ms = ea.elapsed_time(eb) / args.steps
    # the timed steps replay one captured CUDA graph of the whole batched step
    # (--no-graph: eager steps, for profilers that trace kernel launches)
    graph = None
    if not args.no_graph:
        graph = plan.capture(x, X, xa)
        graph.launch(stream)
        torch.cuda.synchronize()

        def step():  # noqa: F811 -- the graph replay replaces the eager step
            graph.launch(stream)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(physical_gpu_index(local))
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed_steps")
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_local = e0.elapsed_time(e1) / 1000.0
    units_local = 2.0 * Mtot * C * args.steps
    t, units = combine_over_ranks(t_local, units_local, world, dev)
    value = units / t / 1e6

    # --- roofline of the interpolation kernels (device buffers, same plan) ---
    ip = plan.lib.mirt_nufft_interp_plan(plan.handle)
    import ctypes as Cc
    grid = torch.randn((plan.nslice,) + (w["K"],) * D + (C,), dtype=torch.complex64, device=dev)
    sptr = Cc.c_void_p(stream.cuda_stream)
    reps = 5

    def timed(fn, name):
        fn()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push(name)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1000.0 / reps

    from mirt_b200._lib import check
    t_gather = timed(lambda: check(plan.lib.mirt_interp_plan_forward(
        ip, Cc.c_void_p(grid.data_ptr()), Cc.c_void_p(X.data_ptr()), sptr)), "roofline_gather")
    t_spread = timed(lambda: check(plan.lib.mirt_interp_plan_adjoint(
        ip, Cc.c_void_p(X.data_ptr()), Cc.c_void_p(grid.data_ptr()), sptr)), "roofline_spread")
    nk = w["K"] ** D
    B = 8.0 * C * nk * plan.nslice + 8.0 * C * Mtot + 4.0 * D * Mtot
    peak, peak_kind = measured_peak()
    dom, tdom = ("spread", t_spread) if t_spread >= t_gather else ("gather", t_gather)
    achieved = B / tdom / 1e9
    variant = {"spread": "sweep" if tuned.get("spread_sweep", 0) != 0 else "tiled",
               "gather": "tma" if tuned.get("gather_tma", 0) else "plain"}
    rows, staged = tuned.get("spread_sweep_rows", 1), tuned.get("spread_staged", 0)
    if D == 3:
        sweep_kernel = "spread_sweep3_kernel"
    elif staged == 2:
        sweep_kernel = f"spread_sweep2s_kernel rows={rows} (caller-order samples)"
    elif staged == 1:
        sweep_kernel = f"sweep_order_kernel + spread_sweep2s_kernel rows={rows}"
    else:
        sweep_kernel = f"sweep_order_kernel + spread_sweep_kernel rows={rows}"
    tma_coils = 16 if tuned.get("gather_tma", 0) == 2 else 32
    kernels = {"gather": (f"gather_tma_kernel ({tma_coils}-coil tiles)" if variant["gather"] == "tma"
                          else "gather_kernel"),
               "spread": (sweep_kernel if variant["spread"] == "sweep"
                          else "spread_kernel (+ spread_reduce_kernel)")}
    traffic, traffic_src = traffic_from_profiles(args.workload, kernels[dom])
    roof = {"bound": "hbm", "kernel": kernels[dom], "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": traffic, "traffic_source": traffic_src,
            "algorithmic_bytes": B,
            "gather": {"ms": 1e3 * t_gather, "GBps": B / t_gather / 1e9,
                       "frac": B / t_gather / 1e9 / peak},
            "spread": {"ms": 1e3 * t_spread, "GBps": B / t_spread / 1e9,
                       "frac": B / t_spread / 1e9 / peak}}
    del grid

    # --- e2e through the host-buffer C ABI ---
    e2e = None
    if not args.no_e2e:
        xh = torch.empty(plan.image_shape, dtype=torch.complex64, pin_memory=True)
        Xh = torch.empty(plan.sample_shape, dtype=torch.complex64, pin_memory=True)
        xh.copy_(x)
        xhn, Xhn = xh.numpy(), Xh.numpy()
        xa_h = torch.empty(plan.image_shape, dtype=torch.complex64, pin_memory=True).numpy()
        ke = max(1, min(args.steps, 5))
        plan.forward_host(xhn, out=Xhn)
        plan.adjoint_host(Xhn, out=xa_h)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            plan.forward_host(xhn, out=Xhn)
            plan.adjoint_host(Xhn, out=xa_h)
        te = time.perf_counter() - t0
        if world > 1:
            tt = torch.tensor([te], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt.item())
        nbx, nbX = xhn.nbytes, Xhn.nbytes
        e2e = {"value": (2.0 * Mtot * C * ke * world) / te / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": nbx + nbX, "d2h_bytes_per_step": nbX + nbx}

    # --- CPU baseline (rank 0, N = 1 only) ---
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = CpuReference(w, om, moff, n_shift)
        v, ns, u, tc = ref.timed_sample(img_np, target_s=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
               "sample": f"{ns} of {plan.nslice} slices, forward + adjoint, {C} coils "
                         f"({u:.3g} sample-coils in {tc:.1f} s)"}
        # one core: the reference's own behaviour (its table code has no threads)
        ref1 = CpuReference(w, om, moff, n_shift, threads=1)
        c1 = 1 if D == 3 else None         # the kooshball: one coil of the slice
        v1, ns1, u1, tc1 = ref1.timed_sample(img_np, target_s=args.cpu_seconds / 2, max_slices=1,
                                             coils=c1)
        cpu["one_core"] = {"value": v1, "unit": UNIT, "cores": 1,
                           "sample": f"{ns1} slice, forward + adjoint, {c1 or C} coil(s) "
                                     f"({u1:.3g} sample-coils in {tc1:.1f} s)"}

    # the library's own launches per forward + adjoint (FFT passes or, with cuFFT,
    # the deapodise / transpose / crop kernels; gather; spread), cuFFT not counted
    fcfg = plan.fft_config()
    launches_per_step = fcfg["launches_forward"] + fcfg["launches_adjoint"]
    cg = None
    if rank == 0 and world == 1 and not args.no_cg and w["D"] == 2:
        cg = run_cgsense(args)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 (f32 arithmetic, f64 table-index selection)", "data": "synthetic",
            "config": {"workload": describe(args.workload, w), "samples_per_rank": Mtot,
                       "coils": C, "slices_per_rank": plan.nslice,
                       "l2": "inputs larger than L2; no flush",
                       "launch": tuned, "autotune_s": round(t_tune, 2),
                       "step": ("eager forward + adjoint of the batch" if args.no_graph
                                else "one CUDA graph launch (forward + adjoint of the batch)"),
                       "adjoint_order": ("shared-memory atomics (not bitwise reproducible)"
                                         if tuned.get("spread_atomic") else
                                         "fixed (bitwise reproducible)"),
                       "eager_ms_per_step": eager_ms,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps, "clocks": clk,
            "cg_sense": cg,
        }
        print(json.dumps(line), flush=True)
    if graph is not None:
        graph.close()
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# batched CG-SENSE: time to NRMSE 1e-3, learned density compensation vs plain
# ---------------------------------------------------------------------------
def _first_below(nr, ms, tol):
    """(device ms, iterations) until every problem of the group has NRMSE <=
    tol, or (None, None); nr [it + 1, S], ms [it]."""
    ok = np.all(nr <= tol, axis=1)
    if ok[0]:
        return 0.0, 0
    hit = np.nonzero(ok)[0]
    if len(hit) == 0:
        return None, None
    i = int(hit[0])
    return float(ms[i - 1]), i


def run_cgsense(args):
    """64 uneven 2D problems (N in {128, 192, 256}, 8-32 coils, golden-angle
    radial at R = 4, 30 dB noise, quadratic Reg1 with beta = 2^-8 trace
    scale), grouped by (N, coils) into batched plans.  Per group: a reference
    solution, then five ways to it, each timed with CUDA events until every
    problem has NRMSE <= 1e-3 (density-compensation and warm-start time
    included; plan and Toeplitz set-up reported apart):
      plain             qpwls_pcg1 from zero (precon = 1), NUFFT pair per iteration
      precon_only       the same with the circulant preconditioner
      learned           learned DCF (features + MLP + PSF scale) warm start + preconditioner
      precon_toeplitz   circulant preconditioner on the Toeplitz normal equations
                        (qpwls_pcg2), from zero: the Gram form without the learned part
      learned_toeplitz  the learned warm start on the Toeplitz normal equations
      pipe              Pipe-Menon DCF (30 updates) warm start + preconditioner
      learned_precon    from zero, the circulant preconditioner built from the learned DCF
                        (G' diag(w^2) G, floored; the learned weights and the preconditioner's
                        kernel built inside the timed region), NUFFT pair per iteration
      learned_precon_blend  the same, blended half and half with the unweighted one"""
    import torch

    import mirt_b200 as mb
    from mirt_b200 import learned_dcf as ld
    from mirt_b200 import sense as ms
    from mirt_b200 import workloads as wl

    tol = 1e-3
    modes = ("plain", "precon_only", "learned", "precon_toeplitz", "learned_toeplitz", "pipe",
             "learned_precon", "learned_precon_blend")
    rng = np.random.default_rng(5)
    probs = wl.cgsense_problems(args.cg_problems, rng)
    groups = {}
    for i, p in enumerate(probs):
        groups.setdefault((p["N"], p["C"]), []).append(i)
    model = ld.LearnedDCF.pretrained()
    model.predict(wl.ga_radial(8, 64))   # first-call set-up (kernel attributes) outside the timing
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(st)
        return e

    tot = {k: 0.0 for k in modes}
    reached = {k: True for k in modes}
    per = []
    setup_s = 0.0
    for (N, C), idx in sorted(groups.items()):
        oms = [probs[i]["om"] for i in idx]
        moff = np.concatenate([[0], np.cumsum([len(o) for o in oms])]).astype(np.int64)
        om = np.concatenate(oms)
        K = 2 * N
        t0 = time.perf_counter()
        G = mb.NufftPlan(om, (N, N), (6, 6), (K, K), n_shift=(N / 2, N / 2), Ld=1024, ncol=C,
                         slice_moff=moff)
        G1 = mb.NufftPlan(om, (N, N), (6, 6), (K, K), n_shift=(N / 2, N / 2), Ld=1024, ncol=1,
                          slice_moff=moff)
        sens = torch.from_numpy(np.stack([probs[i]["sens"] for i in idx])).cuda()
        A = ms.SenseSystem(G, sens, ms.trace_beta(np.diff(moff), sens)).toeplitz()
        torch.cuda.synchronize()
        setup_s += time.perf_counter() - t0
        xt = torch.from_numpy(np.stack([probs[i]["xtrue"] for i in idx])).cuda()
        y = A.forward(xt)
        g = torch.Generator(device="cuda").manual_seed(N * 100 + C)
        noise = torch.randn(y.shape, dtype=torch.complex64, device="cuda", generator=g)
        for s in range(len(idx)):
            a, b = int(moff[s]), int(moff[s + 1])
            noise[a:b] *= y[a:b].norm() / noise[a:b].norm() * 10 ** (-30 / 20)
        y = (y + noise).contiguous()
        om_d = torch.from_numpy(om).cuda()
        xref = torch.zeros(A.image_shape, dtype=torch.complex64, device="cuda")
        A.pcg(xref, y, args.cg_ref, precon=True)
        # untimed first calls of this group's sizes and of every torch op used
        # below (device buffers come from the library's caching allocator
        # afterwards), like the plan set-up
        A.warm_start(y, W=model.predict(om_d, slice_moff=moff).to(torch.float32))
        A.warm_start(y, W=mb.dcf_pipe(G1, niter=0, thresh=0.0).to(torch.float32))
        A.precon_dcf(model.predict(om_d, slice_moff=moff), 0.0)
        torch.zeros_like(xref)
        torch.cuda.synchronize()
        res = {"N": N, "coils": C, "problems": len(idx)}
        # the learned weights' two parts timed apart (CUDA events): features, then
        # the MLP on the tensor cores and, for comparison, on the FP32 pipes
        e_a = ev()
        feat = ld.dcf_features(om_d, (model.K, model.K), moff)
        e_b = ev()
        model.mlp.infer(feat, model.mu, model.sigma)
        e_c = ev()
        model.mlp.set_tensor_cores(False)
        e_d = ev()
        model.mlp.infer(feat, model.mu, model.sigma)
        e_e = ev()
        model.mlp.set_tensor_cores(True)
        torch.cuda.synchronize()
        res.update({"samples": int(moff[-1]), "dcf_features_ms": e_a.elapsed_time(e_b),
                    "mlp_tensor_core_ms": e_b.elapsed_time(e_c),
                    "mlp_fp32_pipes_ms": e_d.elapsed_time(e_e)})
        del feat
        for mode in modes:
            e0 = ev()
            if mode in ("plain", "precon_only", "precon_toeplitz"):
                x = torch.zeros_like(xref)
            elif mode.startswith("learned_precon"):
                w = model.predict(om_d, slice_moff=moff)
                e_p = ev()
                A.precon_dcf(w, 1.0 if mode == "learned_precon" else 0.5)
                e_q = ev()
                x = torch.zeros_like(xref)
            else:
                # the warm start's per-problem least-squares scale absorbs any
                # scale of the weights: no PSF scaling or normalisation here
                if mode == "pipe":
                    w = mb.dcf_pipe(G1, niter=29, thresh=0.0)
                else:
                    w = model.predict(om_d, slice_moff=moff)
                x = A.warm_start(y, W=w.to(torch.float32))
            e1 = ev()
            nr, tms = A.pcg(x, y, args.cg_iters, precon=(mode != "plain"),
                            gram=mode.endswith("_toeplitz"), xref=xref, timing=True)
            torch.cuda.synchronize()
            pre = e0.elapsed_time(e1)
            t, it = _first_below(nr, tms, tol)
            res[mode] = {"s": None if t is None else (pre + t) / 1e3, "setup_s": pre / 1e3,
                         "iters": it, "ms_per_iter": float(tms[-1] / len(tms)),
                         "nrmse_start": float(nr[0].max()), "nrmse_end": float(nr[-1].max())}
            if mode.startswith("learned_precon"):
                res[mode]["precon_build_ms"] = e_p.elapsed_time(e_q)
                A.precon_dcf(w, 0.0)         # the unweighted preconditioner again (untimed)
        for k in modes:
            if res[k]["s"] is None:
                reached[k] = False
            else:
                tot[k] += res[k]["s"]
        per.append(res)
        A.close()
        del G, G1
    out = {"metric": "CG-SENSE s to NRMSE 1e-3 (every problem of the batch)",
           "problems": args.cg_problems, "groups": len(per), "max_iters": args.cg_iters}
    for k in modes:
        out[f"{k}_s"] = tot[k] if reached[k] else None
    out.update({
        "dcf_features_ms": sum(r["dcf_features_ms"] for r in per),
        "mlp_tensor_core_ms": sum(r["mlp_tensor_core_ms"] for r in per),
        "mlp_fp32_pipes_ms": sum(r["mlp_fp32_pipes_ms"] for r in per),
        "plan_and_toeplitz_setup_s": setup_s,
        "reference": f"{args.cg_ref} preconditioned CG iterations from zero (FP32 operators, "
                     "FP64 inner products; within 1e-4 of the FP64 solution on the parity cases)",
        "per_group": per})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mirt", choices=["mirt", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--sweep-config", default="",
                    help="SEGMENTS,ROWS[,STAGED[,DENSE]]: fix the row sweep after autotuning "
                         "(for captures)")
    ap.add_argument("--gather-tma", type=int, default=None, choices=[0, 1, 2],
                    help="fix the gather after autotuning: 0 plain, 1 TMA tiles of 32 coils, "
                         "2 of 16 coils (for captures)")
    ap.add_argument("--no-graph", action="store_true",
                    help="time eager steps instead of a CUDA-graph replay (for profiling)")
    ap.add_argument("--spread", default="auto", choices=["auto", "sweep", "tiled"],
                    help="spread variant: the autotuner's choice, or the row sweep / tiled spread")
    ap.add_argument("--nondeterministic", action="store_true",
                    help="let the spread add with shared-memory atomics (not bitwise reproducible)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cg", action="store_true", help="skip the CG-SENSE comparison")
    ap.add_argument("--cg-problems", type=int, default=64)
    ap.add_argument("--cg-iters", type=int, default=60)
    ap.add_argument("--cg-ref", type=int, default=300)
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, w)
    return run_gpu(args, w)


if __name__ == "__main__":
    sys.exit(main())
