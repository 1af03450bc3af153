#!/usr/bin/env python
"""Benchmark of the Toeplitz SENSE normal operator (A^H A), the NUFFT pair and CG.

Workload (default, one GPU): 160^3 complex64 image, 32 coils, 3-D cones-like spirals with 24000
interleaves x 256 samples (6,144,000 points), |k|^2 density compensation, Kaiser-Bessel width 6,
upsampling 2. Seeded synthetic data, built on the host.

A "step" is one A^H A apply (x -> sum_c conj(S_c) T(S_c x)), the body of the CG loop. `value` is
applies/s over all ranks with the inputs resident in HBM; `e2e` is the same apply through the
public operator with the image copied in from pinned host memory and the result copied back
inside the timed region. The NUFFT type-1 / type-2 throughput (Msamp/s = M * coils / s) and the
graph-captured 20-iteration CG recon rate are reported beside it.

Multi-GPU (torchrun): every rank runs its own replica (frames are independent; no collective
on the data path), so scaling is weak and `value` sums the ranks' work over the slowest rank's
time.

--impl reference times the reference-side CPU implementation (the oracle restatement of the
straight Toeplitz SENSE normal operator, cpp/corelib/lib/fft/nufft.cppm:448-479 +
cpp/corelib/lib/mri/normal.cppm:65-88, multithreaded FFT; one full apply over every coil per
step, with the Toeplitz kernel built by the FP64 gridding oracle) on rank 0.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "A^HA applies/s, NUFFT Msamp/s; batched vs looped CG recons/s @1e-5 rel err"
MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"


# ---------------------------------------------------------------------------------------------
# workload

WORKLOADS = {
    # name: (image shape, coils, trajectory kind, (interleaves, samples), width, dcf, cg iterations)
    "cones160": ((160, 160, 160), 32, "cones", (24000, 256), 6, True, 20),
    "radial64": ((64, 64, 64), 8, "radial", (1024, 128), 4, False, 10),
    # profiling sizes: pass buffers larger than L2 (126 MB), a few GB on the device in total
    "radial96": ((96, 96, 96), 16, "radial", (2048, 192), 6, False, 10),
    "prof160": ((160, 160, 160), 8, "cones", (6000, 256), 6, True, 20),
    "prof96c32": ((96, 96, 96), 32, "radial", (4096, 192), 6, False, 10),
}


def make_workload(name: str):
    from hastycucompute_b200 import synthetic

    shape, C, kind, (ni, ns), w, use_dcf, iters = WORKLOADS[name]
    if kind == "cones":
        coords = synthetic.cones_spiral(ni, ns)
    else:
        coords = synthetic.golden_means_radial(ni, ns)
    dcf = synthetic.dcf_k2(coords) if use_dcf else None
    smaps = synthetic.coil_maps(C, shape)
    x = synthetic.image(shape)
    return dict(name=name, shape=shape, C=C, coords=coords, dcf=dcf, smaps=smaps, x=x, w=w, iters=iters,
                M=coords.shape[1])


def peaks():
    if MEASURED_PEAKS.exists():
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ---------------------------------------------------------------------------------------------
# distributed plumbing

def dist_setup(use_gpu: bool):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl" if use_gpu else "gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, world: int, device) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# reference arm: CPU restatement on the host cores

def run_reference(args, wl_name: str):
    """The reference-side CPU path, timed on the host cores: the Toeplitz kernel built by the FP64
    gridding oracle (cpp/corelib/lib/fft/nufft.cppm:386-441 restated, untimed set-up), then per
    step one full straight Toeplitz SENSE normal apply over every coil (nufft.cppm:448-479 +
    cpp/corelib/lib/mri/normal.cppm:65-88) in complex64 with torch's multithreaded CPU FFT."""
    world, rank, _ = dist_setup(False)
    if rank != 0:
        return 0
    import torch
    from oracle import toeplitz as otp

    wl = make_workload_cpu_only(wl_name)
    shape, C = wl["shape"], wl["C"]
    cores = len(os.sched_getaffinity(0))
    torch.set_num_threads(cores)
    t0 = time.perf_counter()
    K = otp.toeplitz_kernel(list(wl["coords"]), shape, wl["dcf"], w=wl["w"]).astype(np.complex64)
    t_kernel = time.perf_counter() - t0
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        otp.sense_normal(wl["x"], wl["smaps"], K, dtype=np.complex64, fast=True)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    per_apply = statistics.mean(times)
    value = 1.0 / per_apply
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "applies/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_apply * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(wl),
        "cpu_baseline": {"value": value, "unit": "applies/s", "cores": cores, "kind": "port",
                         "sample": f"every step one full apply over all {C} coils (straight Toeplitz SENSE normal, "
                                   f"complex64, torch CPU FFT on {cores} threads); Toeplitz kernel built by the FP64 "
                                   f"gridding oracle in {t_kernel:.1f} s, untimed"},
        "e2e": {"value": value, "unit": "applies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def make_workload_cpu_only(name):
    return make_workload(name)


def workload_config(wl):
    return {
        "workload": f"toeplitz_sense_normal_{wl['name']}",
        "image": list(wl["shape"]), "coils": wl["C"], "samples": int(wl["M"]), "kernel": "kaiser-bessel",
        "kernel_width": wl["w"], "upsampfac": 2.0, "dcf": "|k|^2" if wl["dcf"] is not None else "none",
        "cg_iterations": wl["iters"], "parallelism": "replicas (one frame per rank)",
        "l2": "inputs larger than L2 (coil maps + workspace >> 126 MB)",
    }


# ---------------------------------------------------------------------------------------------
# our arm

# DRAM traffic / algorithmic bytes of the fused pass P3 from one ncu capture at 160^3 x 8 coils
# (1.310864 GB read + 0.994955 GB written for 2.359296 GB algorithmic); traffic and algorithmic
# bytes both grow with (coils + 1), so the ratio carries over.
P3_TRAFFIC_RATIO = (1.310864e9 + 0.994955e9) / 2.359296e9


def aha_bytes(n: int, C: int, dim: int = 3) -> dict:
    """Algorithmic HBM bytes per pass of one fused apply (c64 = 8 B, n voxels, C coils)."""
    if dim == 3:
        return {"toeplitz P1": 8 * n * (3 * C) + 8 * n, "toeplitz P2": 8 * n * 6 * C,
                "toeplitz P3": 8 * n * 8 * C + 8 * n * 8, "toeplitz P4": 8 * n * 6 * C,
                "toeplitz P5 sense": 8 * n * 3 * C + 8 * n}
    return {}


def run_ours(args, wl_name: str):
    import torch

    world, rank, local = dist_setup(True)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import _lib

    wl = make_workload(wl_name)
    shape, C, M, w = wl["shape"], wl["C"], wl["M"], wl["w"]
    n = int(np.prod(shape))
    coords = [torch.from_numpy(np.ascontiguousarray(c)).to(dev) for c in wl["coords"]]
    dcf = torch.from_numpy(wl["dcf"]).to(dev) if wl["dcf"] is not None else None
    smaps = torch.from_numpy(wl["smaps"]).to(dev)
    x = torch.from_numpy(wl["x"]).to(dev)

    t0 = time.perf_counter()
    K = hb.build_toeplitz_kernel(coords, shape, dcf, kernel_width=w)
    torch.cuda.synchronize()
    t_kernel = time.perf_counter() - t0
    op = hb.NormalTT1Op(K, smaps)
    out = torch.empty_like(x)

    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        op.apply(x, out)
    torch.cuda.synchronize()

    # ---- timed region: K applies, inputs resident -----------------------------------------
    _lib.timing_enable(True)
    _lib.timing_read()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            op.apply(x, out)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    per_kernel, launches = _lib.timing_read()
    _lib.timing_enable(False)
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, world, dev)
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)

    # roofline of the dominant kernel
    hbm_peak, peak_kind = peaks()
    bytes_per = aha_bytes(n, C, len(shape))
    kname = max(per_kernel, key=per_kernel.get)
    k_ms = per_kernel[kname] / args.steps
    algo = bytes_per.get(kname, 0)
    achieved = algo / (k_ms / 1e3) / 1e9
    traffic = round(algo * P3_TRAFFIC_RATIO) if kname == "toeplitz P3" else None
    roofline = {"kernel": kname, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(achieved / hbm_peak, 4), "peak_kind": peak_kind,
                "traffic": traffic, "traffic_source": "ncu dram bytes at 160^3 x 8 coils, scaled by (coils+1)",
                "algorithmic_bytes": algo, "avg_ms": round(k_ms, 4),
                "share": round(per_kernel[kname] / sum(per_kernel.values()), 4)}
    apply_bytes = 8 * n * (26 * C + 10)
    aha_roof = {"bytes_model": apply_bytes, "achieved_gbs": round(apply_bytes / (ms_step / 1e3) / 1e9, 1),
                "frac": round(apply_bytes / (ms_step / 1e3) / 1e9 / hbm_peak, 4),
                "per_kernel_ms": {k: round(v / args.steps, 4) for k, v in per_kernel.items()}}

    # ---- e2e: host image in, host result out, through the public operator ------------------
    # every step copies its image in from pinned host memory and its result out; the headline
    # runs them through hb.HostPipeline (copies of neighbouring steps overlap the apply), the
    # serial figure issues copy, apply, copy back to back on one stream
    xh = torch.from_numpy(wl["x"]).pin_memory()
    ohs = [torch.empty_like(xh).pin_memory() for _ in range(2)]
    xd = torch.empty_like(x)
    for _ in range(2):
        xd.copy_(xh, non_blocking=True)
        op.apply(xd, out)
        ohs[0].copy_(out, non_blocking=True)
    torch.cuda.synchronize()
    barrier(world)
    e0.record(stream)
    for _ in range(args.steps):
        xd.copy_(xh, non_blocking=True)
        op.apply(xd, out)
        ohs[0].copy_(out, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    serial_ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    pipe = hb.HostPipeline(lambda a, b: op.apply(a, b), tuple(x.shape), dev)
    pipe.run([xh] * 2, ohs)
    torch.cuda.synchronize()
    barrier(world)
    e0.record(stream)
    pipe.run([xh] * args.steps, [ohs[i & 1] for i in range(args.steps)], compute=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    e2e = {"value": world * args.steps / (e2e_ms / 1e3), "unit": "applies/s",
           "h2d_bytes_per_step": xh.numel() * 8, "d2h_bytes_per_step": ohs[0].numel() * 8,
           "mode": "hb.HostPipeline: H2D of step i+1 and D2H of step i-1 overlap the apply of step i",
           "serial_value": round(world * args.steps / (serial_ms / 1e3), 3)}

    extra = {}
    solver = b = None
    # ---- NUFFT pair ----------------------------------------------------------------------------
    if not args.no_nufft:
        extra["nufft"] = bench_nufft(args, hb, _lib, coords, wl, dev, stream, hbm_peak)
    # ---- CG recon, graph captured --------------------------------------------------------------
    if not args.no_cg:
        solver = hb.CGSolver(lambda v, o: op.apply(v, o), shape, dev, max_iter=wl["iters"], tol=0.0, graph=True)
        b = out.clone()
        solver.solve(torch.zeros_like(x), b)  # capture + warm
        torch.cuda.synchronize()
        e0.record(stream)
        reps = 2
        for _ in range(reps):
            solver.solve(torch.zeros_like(x), b)
        e1.record(stream)
        torch.cuda.synchronize()
        cg_ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / reps
        extra["cg"] = {"recons_per_s": round(world * 1e3 / cg_ms, 3), "iterations": wl["iters"],
                       "ms_per_recon": round(cg_ms, 3), "graph_captured": True}

    # ---- accuracy of the timed apply: coil subset against the FP64 oracle ------------------------
    acc = {}
    if rank == 0 and not args.no_check:
        acc = check_accuracy(hb, wl, K, dev)

    # ---- CPU baseline (rank 0, N = 1 only) ------------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl, K)

    # the remaining sections measure other workloads: release this workload's device state first
    # (operator, workspace, kernel, maps, captured CG, copy pipeline) so they start on a clean device
    del op, K, smaps, x, out, coords, dcf, pipe, xd, solver, b
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    # ---- batched multi-frame recon vs per-frame plain-operator loop ----------------------------
    if not args.no_frames:
        extra["frames"] = bench_frames(args, hb, dev, stream, world, rank)
        torch.cuda.empty_cache()

    # ---- configurations 0, 3 and 4 at their own sizes -------------------------------------------
    if not args.no_configs and rank == 0:
        extra["configs"] = bench_configs(args, hb, dev, stream)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "applies/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(wl), "e2e": e2e,
            "gpu_launches": launches, "roofline": roofline, "aha_roofline": aha_roof,
            "cpu_baseline": cpu, "clocks": clk.summary(), "setup": {"toeplitz_kernel_s": round(t_kernel, 3)},
            "accuracy": acc,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def bench_nufft(args, hb, _lib, coords, wl, dev, stream, hbm_peak):
    import torch
    shape, C, M, w = wl["shape"], wl["C"], wl["M"], wl["w"]
    opts = hb.NufftOpts(nmodes=shape, ntransf=C, kernel_width=w)
    p2 = hb.NufftPlan(hb.NufftType.TYPE_2, opts)
    p2.set_interp_kernel(args.interp_kernel)
    p2.setpts(coords)
    f = torch.from_numpy(wl["smaps"]).to(dev) * torch.from_numpy(wl["x"]).to(dev)[None]
    y = torch.empty((C, M), dtype=torch.complex64, device=dev)
    p1 = hb.NufftPlan(hb.NufftType.TYPE_1, opts)
    p1.setpts(coords)
    g = torch.empty_like(f)
    res = {}
    nf = p1.info().fine
    n_os = int(np.prod(nf))
    d = len(shape)
    for name, plan, a, b in (("type2", p2, f, y), ("type1", p1, y, g)):
        for _ in range(2):
            plan.execute(a, b)
        torch.cuda.synchronize()
        _lib.timing_enable(True)
        _lib.timing_read()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(3, args.steps // 4)
        e0.record(stream)
        for _ in range(reps):
            plan.execute(a, b)
        e1.record(stream)
        torch.cuda.synchronize()
        pk, _ = _lib.timing_read()
        _lib.timing_enable(False)
        ms = e0.elapsed_time(e1) / reps
        res[name] = {"msamp_per_s": round(M * C / (ms / 1e3) / 1e6, 1), "ms": round(ms, 3),
                     "per_kernel_ms": {k: round(v / reps, 4) for k, v in pk.items()}}
        gk = "interp" if name == "type2" else "spread"
        if gk in pk:
            kms = (pk[gk] + pk.get("spread_dense", 0.0)) / reps if gk == "spread" else pk[gk] / reps
            algo = 4 * d * M + C * (8 * M + 8 * n_os)
            res[name]["gridding_roofline"] = {"kernel": gk, "algorithmic_bytes": algo,
                                              "achieved_gbs": round(algo / (kms / 1e3) / 1e9, 1),
                                              "frac": round(algo / (kms / 1e3) / 1e9 / hbm_peak, 4),
                                              "avg_ms": round(kms, 4)}
    # spot checks against the FP64 NUDFT (bounded: 48 points / 48 modes)
    from oracle import nudft
    rng = np.random.default_rng(4)
    pts = rng.choice(M, 48, replace=False)
    f_np = f[:2].cpu().numpy()
    y_ref = nudft.type2_at(wl["coords"], f_np, pts, sign=-1)
    y_got = y[:2].cpu().numpy()[:, pts]
    res["type2"]["rel_err_vs_nudft"] = float(np.linalg.norm(y_got - y_ref) / np.linalg.norm(y_ref))
    idx = np.stack([rng.integers(0, s, 48) for s in shape], axis=1)
    y_np = y[:1].cpu().numpy()
    g_ref = nudft.type1_at(wl["coords"], y_np, shape, idx, sign=1)
    g_got = g[:1].cpu().numpy()[(slice(None),) + tuple(idx[:, i] for i in range(d))]
    res["type1"]["rel_err_vs_nudft"] = float(np.linalg.norm(g_got - g_ref) / np.linalg.norm(g_ref))
    if not args.no_check:
        # two of the transforms at full size against the FP64 gridding oracle (same kernel, width,
        # upsampling; multithreaded C spreading / interpolation)
        from oracle import gridding
        res["type2"]["rel_err_vs_fp64_gridding_2_transforms"] = _rel(
            y[:2].cpu().numpy(), gridding.nufft2(list(wl["coords"]), f_np, w=w))
        res["type1"]["rel_err_vs_fp64_gridding_2_transforms"] = _rel(
            g[:2].cpu().numpy(), gridding.nufft1(list(wl["coords"]), y[:2].cpu().numpy(), shape, w=w))
    p1.free()
    p2.free()
    return res


def bench_frames(args, hb, dev, stream, world=1, rank=0, nframes=24, shape=(128, 128, 128), C=16, iters=15, w=4):
    """Batched dynamic recon: frames with ragged golden-means radial trajectories (300-700 spokes x
    128 samples), per-frame Toeplitz kernels, and three recons of the same right-hand sides:
    - batched: one graph-captured CG over all frames (all frames and coils in one launch per pass);
    - Toeplitz loop: a graph-captured CG on the single-frame fused operator, frame after frame;
    - plain loop: CG on the plain NUFFT SENSE operator (type 2 then type 1 per apply), frame after
      frame, with the adjoint's spreading autotuned for the problem;
    - plain batched: the same plain operator over groups of frames, each group one frame-batched
      NUFFT plan pair (one launch per pass over all its frames' points) and one batched CG.
    The per-frame Toeplitz kernels are built frame-batched (build_toeplitz_kernels).
    With several ranks every rank reconstructs its share of the frames (split by sample count) and
    the times are the slowest rank's."""
    import torch
    from hastycucompute_b200 import autotune, synthetic
    from hastycucompute_b200.frames import frame_partition
    rng = np.random.default_rng(3)
    n = int(np.prod(shape))
    spokes = rng.integers(300, 701, nframes)
    ids = frame_partition(nframes, world, rank, [int(v) * 128 for v in spokes])
    F = len(ids)
    frames = [synthetic.golden_means_radial(int(spokes[f]), 128, offset=int(spokes[:f].sum())) for f in ids]
    xs = synthetic.dynamic_images(nframes, shape)[ids[0]: ids[-1] + 1]
    S = torch.from_numpy(synthetic.coil_maps(C, shape)).to(dev)
    dcoords = [[torch.from_numpy(np.ascontiguousarray(c)).to(dev) for c in fc] for fc in frames]
    t0 = time.perf_counter()
    Ks = hb.build_toeplitz_kernels(dcoords, shape, kernel_width=w)
    torch.cuda.synchronize()
    t_kernels = time.perf_counter() - t0
    t0 = time.perf_counter()
    tune = autotune.tune_spread(shape, C, dcoords[0], w, reps=2, use_cache=True)
    t_tune = time.perf_counter() - t0
    # data y_f = A_f (S x_f) + noise, right-hand sides b_f = (1/n) S^H A_f^H y_f (one plan pair,
    # re-pointed per frame)
    b = torch.empty((F, *shape), dtype=torch.complex64, device=dev)
    so = hb.SenseOp(dcoords[0], S, kernel_width=w, scale=1.0 / math.sqrt(n), spread_tuning=tune)
    for i, f in enumerate(ids):
        so.setpts(dcoords[i])
        y = so.forward(torch.from_numpy(xs[i]).to(dev))
        y = y + torch.from_numpy(synthetic.noise(tuple(y.shape), 1e-3 * float(y.abs().max()), seed=2 + f)).to(dev)
        b[i] = so.adjoint(y)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_region(fn):
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3, world, dev)

    # batched
    op = hb.BatchedNormalOp(Ks, S)
    solver = hb.BatchedCGSolver(lambda v, o: op.apply(v, o), F, shape, dev, max_iter=iters, tol=0.0, graph=True)
    x0 = torch.zeros((F, *shape), dtype=torch.complex64, device=dev)
    solver.solve(x0, b)  # capture + warm-up
    t_batched = timed_region(lambda: solver.solve(x0, b))
    xb = solver.x.clone()
    acc = None
    if not args.no_check and rank == 0:
        # frame 0 of the batched recon against the FP64 oracle CG on its own straight operator
        from oracle import toeplitz as otp
        Sn = S.cpu().numpy().astype(np.complex128)
        Kn = Ks[0].cpu().numpy().astype(np.complex128)
        op0 = hb.NormalTT1Op(Ks[0].contiguous(), S)
        sv0 = hb.CGSolver(lambda v, o: op0.apply(v, o), shape, dev, max_iter=iters, tol=0.0, graph=True)
        acc = _cg_stepwise(sv0, lambda v: otp.sense_normal(v, Sn, Kn, fast=True), iters, x0[0], b[0])
        del sv0, op0
    del solver, op
    torch.cuda.empty_cache()
    # per-frame loop of the fused single-frame operator: one operator and one captured CG whose
    # kernel buffer takes each frame's transformed kernel in turn
    kts = [hb.transform_toeplitz_kernel(Ks[i].contiguous()) for i in range(F)]
    op1 = hb.NormalTT1Op(kts[0].clone(), S, transformed=True)
    sv1 = hb.CGSolver(lambda v, o: op1.apply(v, o), shape, dev, max_iter=iters, tol=0.0, graph=True)
    sv1.solve(x0[0], b[0])  # capture + warm-up
    xt = torch.empty_like(xb)

    def toeplitz_loop():
        for i in range(F):
            op1.kernel_t.copy_(kts[i])
            xt[i] = sv1.solve(x0[i], b[i])

    t_tloop = timed_region(toeplitz_loop)
    del sv1, op1, kts
    torch.cuda.empty_cache()
    # per-frame loop with the plain operator (NUFFT type 2 then type 1 per apply): the frame's
    # points are set, then CG runs on that frame
    sv = hb.CGSolver(lambda v, o: o.copy_(so.normal(v)), shape, dev, max_iter=iters, tol=0.0)
    xl = torch.empty_like(xb)

    def plain_loop():
        for i in range(F):
            so.setpts(dcoords[i])
            xl[i] = sv.solve(x0[i], b[i])

    plain_loop()  # warm-up over every frame: the plans' point buffers reach their largest size
    t_loop = timed_region(plain_loop)
    del sv
    # frame-batched plain operator: groups of frames share one NUFFT plan pair (every pass of a
    # type 2 / type 1 covers the group's points in one launch) and one CG over the group's frames;
    # the group is bounded by the plans' grids (about 3.2 GB per frame and plan at 128^3 x 16 coils)
    G = max(g for g in range(1, min(F, 6) + 1) if F % g == 0)
    bso = hb.BatchedSenseOp([dcoords[i] for i in range(G)], S, kernel_width=w, scale=1.0 / math.sqrt(n),
                            spread_tuning=tune)
    bsv = hb.BatchedCGSolver(lambda v, o: o.copy_(bso.normal(v)), G, shape, dev, max_iter=iters, tol=0.0)
    xpb = torch.empty_like(xb)

    def plain_batched():
        for g0 in range(0, F, G):
            bso.setpts([dcoords[i] for i in range(g0, g0 + G)])
            xpb[g0: g0 + G] = bsv.solve(x0[g0: g0 + G], b[g0: g0 + G])

    plain_batched()  # warm-up over every group
    t_pb = timed_region(plain_batched)
    pdiff = float(torch.linalg.vector_norm(xpb - xl) / torch.linalg.vector_norm(xl))
    del bsv, bso
    torch.cuda.empty_cache()
    diff = float(torch.linalg.vector_norm(xb - xl) / torch.linalg.vector_norm(xl))
    tdiff = float(torch.linalg.vector_norm(xb - xt) / torch.linalg.vector_norm(xt))
    return {"workload": f"{nframes} frames x {shape[0]}^3, {C} coils, golden-means radial 300-700 spokes x 128, "
                        f"KB w={w}, {iters} CG iterations",
            "samples_per_frame": [int(v) * 128 for v in spokes], "ranks": world,
            "batched_recons_per_s": round(nframes / t_batched, 3), "batched_s": round(t_batched, 3),
            "toeplitz_looped_recons_per_s": round(nframes / t_tloop, 3), "toeplitz_looped_s": round(t_tloop, 3),
            "plain_looped_recons_per_s": round(nframes / t_loop, 3), "plain_looped_s": round(t_loop, 3),
            "plain_batched_recons_per_s": round(nframes / t_pb, 3), "plain_batched_s": round(t_pb, 3),
            "plain_batched_frames_per_plan": G, "plain_batching_gain": round(t_loop / t_pb, 3),
            "plain_batched_vs_plain_looped_rel_diff": pdiff,
            "batching_gain": round(t_tloop / t_batched, 3), "toeplitz_gain": round(t_loop / t_tloop, 3),
            "speedup_vs_plain_loop": round(t_loop / t_batched, 2),
            "batched_vs_toeplitz_looped_rel_diff": tdiff, "batched_vs_plain_looped_rel_diff": diff,
            "frame0_cg_step_rel_err_vs_fp64_oracle": acc,
            "spread_tuning": {k: tune[k] for k in ("kernel", "block", "max_candidates", "ms")},
            "tuning_s": round(t_tune, 2), "toeplitz_kernels_s": round(t_kernels, 3), "graph_captured": True}


def bench_configs(args, hb, dev, stream):
    """Configurations 0, 3 and 4 at their own sizes, bounded to seconds each:
    0: 64^3, 8 coils, golden-means radial 1024 x 128, KB w=4: A^H A applies/s, NUFFT Msamp/s,
       10-iteration graph-captured CG;
    3: 2-D 256^2, 12 coils, 32 variable-density spiral interleaves x 2048, w=4: NUFFT Msamp/s and
       one forward + backward of ||A^H(Ax - y)||^2 + lam * slew through the coordinate-gradient
       kernels (finite-difference agreement is checked in the GPU tests);
    4: 4 volumes of 128^3, 12 coils, 3-D radial 16384 x 128 (2.1 M points) each, 10 unrolled
       Toeplitz SENSE-CG iterations with learnable steps and weights, per-iteration recomputation:
       forward + backward time and peak HBM allocated by torch."""
    import torch
    from hastycucompute_b200 import autograd as ag, synthetic
    from hastycucompute_b200.unrolled import UnrolledCG

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def todev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def nufft_rates(shape, C, dc, w):
        M = dc[0].shape[0]
        opts = hb.NufftOpts(nmodes=shape, ntransf=C, kernel_width=w)
        p2, p1 = hb.NufftPlan(hb.NufftType.TYPE_2, opts), hb.NufftPlan(hb.NufftType.TYPE_1, opts)
        p2.setpts(dc)
        p1.setpts(dc)
        f = torch.randn((C, *shape), dtype=torch.complex64, device=dev)
        y = torch.empty((C, M), dtype=torch.complex64, device=dev)
        g = torch.empty_like(f)
        t2 = timed(lambda: p2.execute(f, y), 10)
        t1 = timed(lambda: p1.execute(y, g), 10)
        p1.free()
        p2.free()
        return round(M * C / (t2 / 1e3) / 1e6, 1), round(M * C / (t1 / 1e3) / 1e6, 1)

    res = {}
    # ---- config 0 --------------------------------------------------------------------------------
    shape, C, w = (64, 64, 64), 8, 4
    dc = [todev(c) for c in synthetic.golden_means_radial(1024, 128)]
    S = todev(synthetic.coil_maps(C, shape))
    x = todev(synthetic.image(shape))
    K = hb.build_toeplitz_kernel(dc, shape, kernel_width=w)
    op = hb.NormalTT1Op(K, S)
    o = torch.empty_like(x)
    aha_ms = timed(lambda: op.apply(x, o), 20)
    t2r, t1r = nufft_rates(shape, C, dc, w)
    b = op(x)
    solver = hb.CGSolver(lambda v, out: op.apply(v, out), shape, dev, max_iter=10, tol=0.0, graph=True)
    cg_ms = timed(lambda: solver.solve(torch.zeros_like(x), b), 3)
    res["config0"] = {"workload": "64^3, 8 coils, golden-means radial 1024 x 128, KB w=4",
                      "aha_applies_per_s": round(1e3 / aha_ms, 1), "type2_msamp_per_s": t2r,
                      "type1_msamp_per_s": t1r, "cg10_recons_per_s": round(1e3 / cg_ms, 2)}
    if not args.no_check:
        # the timed recon against the FP64 oracle CG (cpp/corelib/lib/op/cg.cppm:122-184 restated) on
        # the FP64 straight Toeplitz SENSE normal operator with the same kernel
        from oracle import cg as ocg, toeplitz as otp
        Sn = S.cpu().numpy().astype(np.complex128)
        Kn = K.cpu().numpy().astype(np.complex128)
        A64 = lambda v: otp.sense_normal(v, Sn, Kn, fast=True)
        res["config0"]["cg10_step_rel_err_vs_fp64_oracle"] = _cg_stepwise(solver, A64, 10, torch.zeros_like(x), b)
        x_ref, _ = ocg.conjugate_gradient(A64, b.cpu().numpy(), np.zeros(shape, np.complex64), 10, tol=0.0)
        res["config0"]["cg10_run_rel_diff_vs_fp64_oracle"] = _rel(solver.x.cpu().numpy(), x_ref)
        res["config0"]["aha_rel_err_vs_fp64_oracle"] = _rel(b.cpu().numpy(), otp.sense_normal(
            x.cpu().numpy(), Sn, Kn, fast=True))
    del solver, op, K, S
    # ---- config 3 --------------------------------------------------------------------------------
    shape, C, ninter, ns = (256, 256), 12, 32, 2048
    k0 = synthetic.variable_density_spiral_2d(ninter, ns)
    dc = [todev(c) for c in k0]
    t2r, t1r = nufft_rates(shape, C, dc, w)
    S = todev(synthetic.coil_maps(C, shape))
    xt = todev(synthetic.image(shape))
    pair = ag.NufftPair(shape, C, kernel_width=w)
    kk = todev(k0)
    with torch.no_grad():
        y = ag.nufft_forward(S * xt[None], kk, pair)
    x0 = todev(synthetic.image(shape, seed=5))

    def step():
        xg = x0.clone().requires_grad_(True)
        kg = kk.clone().requires_grad_(True)
        r = ag.nufft_forward(S * xg[None], kg, pair) - y
        gimg = (torch.conj(S) * ag.nufft_adjoint(r, kg, pair)).sum(0)
        k3 = kg.reshape(2, ninter, ns)
        slew = ((k3[:, :, 2:] - 2 * k3[:, :, 1:-1] + k3[:, :, :-2]) ** 2).sum()
        loss = (gimg.abs() ** 2).sum() + 1e-3 * slew
        loss.backward()

    loss_ms = timed(step, 3)
    res["config3"] = {"workload": "2-D 256^2, 12 coils, 32 variable-density spirals x 2048, KB w=4",
                      "type2_msamp_per_s": t2r, "type1_msamp_per_s": t1r,
                      "loss_forward_backward_ms": round(loss_ms, 2)}
    if not args.no_check:
        # gradients of the timed loss against the FP64 gridding oracle of the same loss: the image
        # gradient exactly, 16 coordinate gradients by central differences (h = 1e-4)
        from oracle.loss import SenseLoss
        xg = x0.clone().requires_grad_(True)
        kg = kk.clone().requires_grad_(True)
        r = ag.nufft_forward(S * xg[None], kg, pair) - y
        gimg = (torch.conj(S) * ag.nufft_adjoint(r, kg, pair)).sum(0)
        k3 = kg.reshape(2, ninter, ns)
        slew = ((k3[:, :, 2:] - 2 * k3[:, :, 1:-1] + k3[:, :, :-2]) ** 2).sum()
        ((gimg.abs() ** 2).sum() + 1e-3 * slew).backward()
        ol = SenseLoss(S.cpu().numpy(), y.cpu().numpy(), k0, w=w, lam=1e-3, interleaves=ninter)
        ol.setup(x0.cpu().numpy())
        rng = np.random.default_rng(4)
        M3 = k0.shape[1]
        picks = []
        while len(picks) < 16:
            a, j = divmod(int(rng.integers(0, 2 * M3)), M3)
            if (a, j) not in picks and not ol.crosses_cell(a, j, 1e-4):
                picks.append((a, j))
        gk = kg.grad.cpu().numpy().astype(np.float64)
        fd = np.array([ol.coord_fd(a, j, 1e-4) for a, j in picks])
        res["config3"]["image_grad_rel_err_vs_fp64_oracle"] = _rel(xg.grad.cpu().numpy(), ol.image_grad())
        res["config3"]["coord_grad_rel_err_vs_central_differences"] = _rel(np.array([gk[a, j] for a, j in picks]), fd)
        res["config3"]["coord_grad_check"] = "16 coordinates, h = 1e-4, FP64 gridding oracle loss (64 in the GPU tests)"
    del pair, S
    torch.cuda.empty_cache()
    # ---- config 4 --------------------------------------------------------------------------------
    F, shape, C = 4, (128, 128, 128), 12
    frames = [[todev(c) for c in synthetic.golden_means_radial(16384, 128, offset=16384 * f)] for f in range(F)]
    Ks = hb.build_toeplitz_kernels(frames, shape, kernel_width=w)
    del frames
    S = todev(synthetic.coil_maps(C, shape))
    op4 = hb.BatchedNormalOp(Ks, S)
    xt = todev(synthetic.dynamic_images(F, shape))
    ob = torch.empty_like(xt)
    apply_ms = timed(lambda: op4.apply(xt, ob), 5)
    b4 = op4(xt)
    acc4 = None
    if not args.no_check:
        from oracle import toeplitz as otp
        acc4 = _rel(b4[0].cpu().numpy(), otp.sense_normal(xt[0].cpu().numpy(), S.cpu().numpy().astype(np.complex128),
                                                          Ks[0].cpu().numpy().astype(np.complex128), fast=True))
    net = UnrolledCG(op4, iterations=10, step_init=0.9, lam_init=0.01, checkpoint=True).to(dev)

    def fb():
        net.zero_grad(set_to_none=True)
        loss = ((net(b4) - xt).abs() ** 2).sum()
        loss.backward()

    fb()
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats(dev)
    base = torch.cuda.memory_allocated(dev)
    fb_ms = timed(fb, 1)
    peak = torch.cuda.max_memory_allocated(dev)
    res["config4"] = {"workload": "4 x 128^3, 12 coils, 3-D radial 16384 x 128 per volume, KB w=4, "
                                  "10 unrolled CG iterations, per-iteration recomputation",
                      "aha_applies_per_s_per_volume": round(F * 1e3 / apply_ms, 1),
                      "unrolled_forward_backward_ms": round(fb_ms, 1),
                      "peak_hbm_gb": round(peak / 1e9, 2), "resident_before_gb": round(base / 1e9, 2),
                      "aha_rel_err_vs_fp64_oracle": acc4,
                      "scalar_gradient_check": "tests/test_configs_gpu.py: the 20 learnable scalars at this size "
                                               "vs central differences with two Richardson steps, <= 1e-3"}
    del net, op4, Ks, S
    torch.cuda.empty_cache()
    return res


def _cg_stepwise(solver, A64, iters, x0, b) -> float:
    """Largest relative error of the device CG's start and of each of its iterations against one
    FP64 iteration of the reference recurrence (oracle.cg.cg_iteration) from the device's own state.
    The whole run is also reported against the FP64 run: on ill-conditioned systems FP32 rounding
    grows along the run, while each step stays at rounding level."""
    from oracle import cg as ocg
    solver.start(x0, b)
    r0 = b.cpu().numpy().astype(np.complex128) - A64(x0.cpu().numpy().astype(np.complex128))
    worst = max(_rel(solver.r.cpu().numpy(), r0), _rel(solver.p.cpu().numpy(), r0))
    for _ in range(iters):
        st = [t.cpu().numpy().astype(np.complex128) for t in (solver.x, solver.r, solver.p)]
        solver.run(1)
        ref = ocg.cg_iteration(A64, *st)
        for t, o in zip((solver.x, solver.r, solver.p), ref[:3]):
            worst = max(worst, _rel(t.cpu().numpy(), o))
    return worst


def _rel(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def check_accuracy(hb, wl, K, dev):
    """Runs the fused apply on a 2-coil subset and compares it with the FP64 oracle apply using
    the same kernel."""
    import torch
    from oracle import toeplitz as otp
    sub = wl["smaps"][:2]
    op2 = hb.NormalTT1Op(K, torch.from_numpy(sub).to(dev))
    got = op2(torch.from_numpy(wl["x"]).to(dev)).cpu().numpy()
    Kn = K.cpu().numpy().astype(np.complex128)
    cores = len(os.sched_getaffinity(0))
    ref = otp.sense_normal(wl["x"], sub, Kn, workers=cores)
    K_ref = otp.toeplitz_kernel(list(wl["coords"]), wl["shape"], wl["dcf"], w=wl["w"])
    return {"aha_rel_err_vs_fp64_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "coils_checked": 2, "toeplitz_kernel_rel_err_vs_fp64_oracle": _rel(Kn, K_ref)}


def cpu_baseline(wl, K):
    """Two full straight Toeplitz SENSE normal applies (every coil) on the host cores with the
    kernel the GPU built, complex64, torch's CPU FFT on all cores; the mean is reported."""
    from oracle import toeplitz as otp
    import torch
    cores = len(os.sched_getaffinity(0))
    torch.set_num_threads(cores)
    Kn = K.cpu().numpy()
    C = wl["C"]
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        otp.sense_normal(wl["x"], wl["smaps"], Kn, dtype=np.complex64, fast=True)
        times.append(time.perf_counter() - t0)
    per_apply = statistics.mean(times)
    return {"value": round(1.0 / per_apply, 5), "unit": "applies/s", "cores": cores, "kind": "port",
            "sample": f"2 full applies over all {C} coils (straight Toeplitz SENSE normal, complex64, torch CPU "
                      f"FFT on {cores} threads), mean {per_apply:.2f} s per apply"}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="cones160")
    ap.add_argument("--no-nufft", action="store_true")
    ap.add_argument("--no-cg", action="store_true")
    ap.add_argument("--no-frames", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--interp-kernel", choices=["auto", "gather", "staged"], default="auto",
                    help="type-2 interpolation kernel of the NUFFT leg (both give bit-identical samples)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args, args.workload)
    return run_ours(args, args.workload)


if __name__ == "__main__":
    sys.exit(main())
