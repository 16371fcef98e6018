"""Benchmark of the PIV hot path: interrogation-area (IA) correlations/s.

Workload (default, --workload vortex2048): the 2048x2048 Float32 Lamb-Oseen
vortex pair with ramp and gain, interSize 32, searchMargin 16, step 8 (64,009
IAs per pair), NSQECC (the reference's default algorithm; --alg zncc for
ZNCC).  --workload shear3d: the 512x512x256 Float32 volume pair (uniform shift
plus du/dz shear), FFTCC, interSize 32^3, searchMargin 16^3, step 16^3 (14,415
IAs).  --workload window256: the vortex pair at interSize 128, searchMargin
64, step 32 (search windows of 256, the coarsest pass of a 3-level refinement
from interSize 32; 3,721 IAs at 2048^2).  One step = one PIV of one image pair.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]

Under torchrun every rank runs an independent replica (the path shards by
image pair with no exchange); the step time is the max over ranks and
``value`` counts the IAs of all ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "IA correlations/s"
UNIT = "IA/s"


def flops_per_ia(cs=64, P=33, IS=32, norm=True, nd=2):
    """Reference-equivalent FLOPs of one IA correlation (unpruned r2c/c2r of
    size cs^nd, conj-multiply, peak scan; +normalisation for ZNCC/NSQECC)."""
    Nc = cs ** nd
    B = (cs // 2 + 1) * cs ** (nd - 1)
    f = 3 * 2.5 * Nc * math.log2(Nc) + 6 * B + P ** nd
    if norm:
        f += 12 * P ** nd + 2 * IS ** nd
    return f


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 50 ms while running.
    Start it before the warm-up (nvidia-smi takes a moment to produce its
    first sample); summary(t0, t1) keeps the samples taken between two
    time.time() marks (the timed region), or all of them if that window
    holds fewer than three."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.idx = gpu_index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0=None, t1=None):
        if self.proc is None or self.out is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        import datetime
        self.out.seek(0)
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[2]), float(parts[3]),
                             {n for n, v in zip(names, parts[6:10]) if v.lower().startswith("active")}))
            except ValueError:
                continue
        window = "timed region"
        sel = [r for r in rows if t0 is None or (t0 - 0.05 <= r[0] <= t1 + 0.05)]
        if len(sel) < 3:
            sel, window = rows, "warm-up and timed region (the timed region held fewer than 3 samples)"
        reasons = set().union(*[r[3] for r in sel]) if sel else set()
        return {"sm_mhz": statistics.median(r[1] for r in sel) if sel else None,
                "sm_max_mhz": max(r[2] for r in sel) if sel else None,
                "samples": len(sel), "window": window, "reasons": sorted(reasons)}


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def max_over_ranks(x, world, device=None):
    """The largest of every rank's x: each rank's device time (or host time)
    of its K steps, so the job's time is the slowest replica's.  Every rank
    must call it, in the same order (one all-reduce)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, steps, seconds):
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank per step for `steps` steps in `seconds` (the max over ranks)."""
    return world * units_per_rank * steps / seconds


class Workload:
    """One bench workload: the image pair, its parameters and its counts."""

    def __init__(self, args):
        from multi_quickpiv_b200 import setPIVParameters, synth
        self.name = args.workload
        if args.workload == "shear3d":
            # 512x512x256 Float32 volumes, uniform shift + du/dz shear, FFTCC, IS 32 SM 16 step 16
            self.i1, self.i2, _ = synth.pair_3d_shear()
            self.alg = "fft"
            self.IS, self.SM, self.step = 32, 16, 16
            self.desc = "shear pair 512x512x256 float32, fft, IS 32 SM 16 step 16"
        elif args.workload == "window256":
            # search windows of 256 (interSize 128, margin 64: the coarsest pass of a 3-level
            # refinement from interSize 32), 2D vortex pair, step 32
            self.i1, self.i2, _ = synth.pair_2d_vortex(shape=(args.size, args.size))
            self.alg = args.alg
            self.IS, self.SM, self.step = 128, 64, 32
            self.desc = f"vortex pair {args.size}x{args.size} float32, {args.alg}, IS 128 SM 64 step 32"
        else:
            self.i1, self.i2, _ = synth.pair_2d_vortex(shape=(args.size, args.size))
            self.alg = args.alg
            self.IS, self.SM, self.step = 32, 16, 8
            self.desc = f"vortex pair {args.size}x{args.size} float32, {args.alg}, IS 32 SM 16 step 8"
        self.nd = self.i1.ndim
        self.params = setPIVParameters(corr_alg=self.alg, interSize=(self.IS,) * self.nd,
                                       searchMargin=(self.SM,) * self.nd, step=(self.step,) * self.nd,
                                       computeSN=False)
        self.params.ndims = self.nd
        self.vf = tuple((n - self.IS) // self.step + 1 for n in self.i1.shape)
        self.n_ia = int(np.prod(self.vf))
        norm = self.alg != "fft"
        self.fft_len = 256 if args.workload == "window256" else 64
        self.flop_per_ia = flops_per_ia(cs=self.fft_len, P=2 * self.SM + 1, IS=self.IS, norm=norm, nd=self.nd)
        npx = int(np.prod(self.i1.shape))
        ii = int(np.prod([n + 1 for n in self.i1.shape])) * 8
        # algorithmic bytes of one pass: both images once, the FP64 integral
        # image of img2^2 once (ZNCC: three), the vectors out
        self.alg_bytes = 2 * npx * 4 + (ii * (3 if self.alg == "zncc" else 1) if norm else 0) + self.n_ia * 8 * self.nd
        self.image_bytes = npx * 4


# ---------------------------------------------------------------------------
def cpu_baseline_sample(wl, budget_s=12.0):
    """The oracle restatement timed on this host on a bounded sample of the
    workload's IAs; returns IA/s, threads used and the sample description."""
    import oracle.cpu_ref as cref
    if not cref.available():
        cref.build()
    return cref.time_sample(wl.i1, wl.i2, wl.alg, budget_s=budget_s, IS=wl.IS, SM=wl.SM, step=wl.step)


def run_reference(args):
    rank, local, world = dist_env()
    if rank != 0:
        return 0
    wl = Workload(args)
    import oracle.cpu_ref as cref
    if not cref.available():
        cref.build()
    K, W = args.steps, args.warmup
    res = None
    times = []
    for it in range(W + K):
        r = cref.time_sample(wl.i1, wl.i2, wl.alg, budget_s=args.ref_budget, IS=wl.IS, SM=wl.SM, step=wl.step)
        if it >= W:
            times.append(r)
        res = r
    vals = [r["value"] for r in times]
    value = statistics.mean(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": 1e3 * wl.n_ia / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.desc, "n_ia_per_pair": wl.n_ia},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["cores"], "kind": res["kind"],
                             "sample": res["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def kernel_launches(wl, chunk3d):
    """Kernels of this library one PIV call launches (counted from the code
    path: integral scans, the fused 2D kernel, or per 3D chunk K3a, its
    merge, K3b, K3c and its merge)."""
    scans = 0
    if wl.alg != "fft":
        per_image = 3 if wl.nd == 2 else 4  # cols, row chunks, row offsets (+ z scan)
        scans = per_image * (3 if wl.alg == "zncc" else 1)
    if wl.nd == 2:
        return scans + 1
    chunks = -(-wl.n_ia // chunk3d)
    return scans + 5 * chunks


def run_ours(args):
    import ctypes as C

    import torch
    import torch.distributed as dist
    rank, local, world = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import multi_quickpiv_b200 as mq
    from multi_quickpiv_b200 import _lib, tune
    ctx = _lib.Context(local)
    wl = Workload(args)
    shape, nd, n_ia = wl.i1.shape, wl.nd, wl.n_ia

    # device-resident inputs (column-major, Julia order)
    d1 = mq.piv._colmajor_torch(torch.from_numpy(wl.i1).to(dev))
    d2 = mq.piv._colmajor_torch(torch.from_numpy(wl.i2).to(dev))
    VF = torch.zeros(tuple(reversed((nd,) + wl.vf)), dtype=torch.float64, device=dev)
    cp = wl.params.to_c()
    dims = (C.c_int64 * 3)(*(list(shape) + [1] * (3 - nd)))
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def step():
        rc = ctx.lib.mqp_piv_device(ctx.handle, C.c_void_p(d1.data_ptr()), C.c_void_p(d2.data_ptr()), None, None,
                                    _lib.MQP_F32, nd, dims, C.byref(cp), C.c_void_p(VF.data_ptr()), None,
                                    C.c_void_p(stream.cuda_stream))
        _lib.check(rc, ctx.handle)

    chunk3d = None
    if nd == 3 and args.chunk3d:
        chunk3d, tuned = args.chunk3d, "fixed by --chunk3d"
        ctx.set_chunk3d(chunk3d, 0)
    elif nd == 3:
        # launch tuning (results never depend on it): IAs per 3D chunk, timed here
        chunk3d, tuned = tune.autotune_chunk3d(ctx, step, stream, candidates=(1024, 2048, 4096, 8192, 16384))
    clk = ClockSampler(local).__enter__()  # sampling from the warm-up on (nvidia-smi starts slowly)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ctx.profile_enable(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_on = time.time()
    for k in range(args.steps):
        flush.fill_(float(k))  # evict the inputs from L2 between steps (not timed)
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    t_off = time.time()
    clk.__exit__()
    if world > 1:
        dist.barrier()
    prof = ctx.profile_read()
    ctx.profile_enable(False)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms), world, dev)
    ms_per_step = total_ms / args.steps
    value = job_rate(world, n_ia, args.steps, total_ms / 1e3)

    # ---- e2e through the public API from pinned host memory ----
    npx = int(np.prod(shape))
    h1p = torch.empty(npx, dtype=torch.float32, pin_memory=True).numpy().reshape(shape, order="F")
    h2p = torch.empty(npx, dtype=torch.float32, pin_memory=True).numpy().reshape(shape, order="F")
    h1p[...] = wl.i1
    h2p[...] = wl.i2
    for _ in range(max(1, args.warmup // 2)):
        mq.PIV(h1p, h2p, wl.params, context=ctx)
    e2e_steps = args.steps if nd == 2 else max(3, args.steps // 10)
    e2e_t = []
    for k in range(e2e_steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        VFh, _ = mq.PIV(h1p, h2p, wl.params, context=ctx)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(e2e_t), world, dev)
    e2e_value = job_rate(world, n_ia, e2e_steps, e2e_s)

    peaks, src = measured_peaks()
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6
    kern_ms = prof["ms_piv"] / max(prof["launches_piv"], 1)
    achieved = wl.flop_per_ia * n_ia / (kern_ms / 1e3)
    traffic = None
    tfile = "piv2d_traffic.json" if nd == 2 else "piv3d_traffic.json"
    if wl.name == "window256":
        tfile = "piv2d_huge_traffic.json"
    try:
        with open(os.path.join(ROOT, "profiles", tfile)) as f:
            tr = json.load(f)
        # measured DRAM bytes of one pass, scaled by interrogation areas
        traffic = tr["dram_bytes_per_launch"] * n_ia / tr["ia_per_launch"]
    except Exception:
        pass
    kname = ("piv2d_kernel (one IA per warp, FFT length 64, search windows staged by TMA)" if nd == 2
             else "k3a_kernel + k3b_kernel + k3c_kernel (all chunks of one pass)")
    if wl.name == "window256":
        kname = "piv2d_huge_kernel (one 256-thread block per IA, FFT length 256)"
    roof = {"bound": "fp32", "kernel": kname, "achieved": achieved / 1e12, "peak": fp32_peak / 1e12,
            "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
            "traffic_unit": f"bytes per pass (ncu dram__bytes_read+write, profiles/{tfile})",
            "algorithmic_bytes_per_launch": wl.alg_bytes,
            "peak_source": f"148 SM x 128 FP32 lanes x 2 x sm_max_mhz from MEASURED_PEAKS.json ({src})",
            "kernel_ms": kern_ms, "algorithmic_flop_per_ia": wl.flop_per_ia,
            "hbm_frac_of_measured": wl.alg_bytes / (kern_ms / 1e3) / (peaks.get("hbm_gbs", 6650) * 1e9)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline_sample(wl)
        except Exception as e:  # reported, never fatal
            cpu = {"value": None, "error": str(e)}
    if rank == 0:
        cfg = {"workload": wl.desc, "n_ia_per_pair": n_ia, "parallelism": f"replicas x{world}",
               "l2": "flushed between steps by a 256 MiB write outside the timed events",
               "compute": "FP32 FFTs, FP64 integral images and normalisation"}
        if chunk3d:
            cfg["chunk3d"] = chunk3d
            cfg["chunk3d_tuning_ms"] = tuned
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": cfg,
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": int(2 * wl.image_bytes),
                        "d2h_bytes_per_step": int(n_ia * nd * 8)},
                "gpu_launches": kernel_launches(wl, chunk3d or 1) * args.steps,
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(t_on, t_off),
                "kernel_ms": {"piv": kern_ms, "integral_scans": prof["ms_integral"] / max(args.steps, 1)}}
    del d1, d2, VF, flush
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line if rank == 0 else None


# ---------------------------------------------------------------------------
# the batched workload: 64 mixed pairs, 3-pass refinement (windows halving)
# ---------------------------------------------------------------------------
def batch_pairs(size_scale=1.0):
    """64 pairs of mixed size and dimensionality; interSize drawn from
    {16, 32, 64} is the coarsest pass's window, halved on each of 3 passes
    (the final pass uses interSize/4, searchMargin interSize/8, step = window)."""
    import multi_quickpiv_b200 as mq
    from multi_quickpiv_b200 import synth
    pairs = []
    for it in synth.batch_mixed(64, size_scale=size_scale):
        nd = it.img1.ndim
        IS = it.interSize // 4
        p = mq.setPIVParameters(corr_alg=it.corr_alg, interSize=(IS,) * nd, searchMargin=(max(IS // 2, 1),) * nd,
                                step=(IS,) * nd, multipass=3, refine=True, computeSN=False)
        pairs.append((it.img1, it.img2, p) + ((it.mask,) if it.mask is not None else ()))
    return pairs


def pass_flops(pairs):
    """Reference-equivalent FLOPs of every pass of every pair (FFT of the
    search-window size per axis, the reference's unpruned convention)."""
    total, n_ia = 0.0, 0
    for pr in pairs:
        shape, p = pr[0].shape, pr[2]
        nd = len(shape)
        for lvl in range(p.multipass):
            sc = 2 ** lvl
            IS, SM = p.interSize[0] * sc, p.searchMargin[0] * sc
            st = p.step[0] * sc
            vf = [(n - IS) // st + 1 if n >= IS else 0 for n in shape]
            n = int(np.prod(vf))
            total += n * flops_per_ia(cs=IS + 2 * SM, P=2 * SM + 1, IS=IS, norm=p.corr_alg != "fftcc", nd=nd)
            n_ia += n
    return total, n_ia


def run_batch_plan_only(args):
    """The batch plan alone (default options, no per-pair comparison, no
    autotuning): K timed replays after W warm-up replays, for profiling."""
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    import torch

    from multi_quickpiv_b200.batch import BatchPlan
    pairs = batch_pairs()
    plan = BatchPlan(pairs)
    s = torch.cuda.current_stream()
    for _ in range(args.warmup):
        plan.run()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(args.steps):
        plan.run()
    b.record(s)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / max(args.steps, 1)
    info = plan.info()
    print(json.dumps({"metric": METRIC, "value": info["total_ia"] / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "config": {"workload": "batch64 plan only (default options, L2 not flushed)",
                                 "launches_per_run": info["launches"]}}), flush=True)
    plan.close()
    return 0


def run_batch(args):
    rank, _, world = dist_env()
    if rank != 0:  # a single-GPU workload: under a multi-rank launch rank 0 runs it alone
        return None
    if args.plan_only:
        run_batch_plan_only(args)
        return None
    import torch

    import multi_quickpiv_b200 as mq
    from multi_quickpiv_b200 import tune
    t0 = time.time()
    pairs = batch_pairs()
    gen_s = time.time() - t0
    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream(dev)
    # plain fused path: one PIV call per pair on device-resident images
    dp = []
    for pr in pairs:
        t1 = mq.piv._colmajor_torch(torch.from_numpy(pr[0]).to(dev))
        t2 = mq.piv._colmajor_torch(torch.from_numpy(pr[1]).to(dev))
        tm = mq.piv._colmajor_torch(torch.from_numpy(np.asarray(pr[3], np.float32)).to(dev)) if len(pr) > 3 else None
        dp.append((t1, t2, pr[2], tm))

    def plain():
        for t1, t2, p, tm in dp:
            mq.PIV(t1, t2, *([tm] if tm is not None else []), p)
    for _ in range(max(1, args.warmup // 2)):
        plain()
    ms_plain = tune.time_ms(plain, s, max(1, args.steps // 4))
    best, tuning, plan = tune.autotune_batch(pairs)
    for _ in range(args.warmup):
        plan.run()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(s)
            plan.run()
            ev[k][1].record(s)
        torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    info = plan.info()
    flops, n_ia = pass_flops(pairs)
    # e2e: every pair's images copied in from pinned host memory, the plan run,
    # every VF read back
    hosts = []
    for k, pr in enumerate(pairs):
        t1, t2 = plan._keep[6 * k], plan._keep[6 * k + 1]
        h1 = torch.empty_like(t1, device="cpu").pin_memory()
        h2 = torch.empty_like(t2, device="cpu").pin_memory()
        h1.copy_(t1)
        h2.copy_(t2)
        hosts.append((h1, h2, t1, t2))
    h2d = sum(h1.numel() * h1.element_size() * 2 for h1, _, _, _ in hosts)
    d2h = sum(VF.numel() * 8 for VF, _ in plan.results())
    e2e = []
    for k in range(max(2, args.steps // 4)):
        torch.cuda.synchronize()
        ta = time.perf_counter()
        for h1, h2, t1, t2 in hosts:
            t1.copy_(h1, non_blocking=True)
            t2.copy_(h2, non_blocking=True)
        plan.run()
        outs = [VF.cpu() for VF, _ in plan.results()]
        e2e.append(time.perf_counter() - ta)
    # the same pairs the way a caller of PIV() would run them without plans:
    # one call per pair from host arrays (copies in, VF/SN out)
    plain_e2e = []
    for k in range(2):
        ta = time.perf_counter()
        for pr in pairs:
            mq.PIV(pr[0], pr[1], *([pr[3]] if len(pr) > 3 else []), pr[2])
        plain_e2e.append(time.perf_counter() - ta)
    peaks, src = measured_peaks()
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6
    value = info["total_ia"] / (ms / 1e3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batch of 64 mixed pairs (2D 512^2-4096x2048, 3D 128^3-256^3), 3-pass refinement, "
                                   "interSize {16,32,64} halving, 25% masked NSQECC",
                       "pairs": len(pairs), "ia_all_passes": info["total_ia"], "generation_s": gen_s,
                       "plan": best, "tuning_ms": tuning, "plan_scratch_bytes": info["scratch_bytes"],
                       "l2": "flushed between steps by a 256 MiB write outside the timed events"},
            "plain_path": {"ms_per_step": ms_plain, "value": info["total_ia"] / (ms_plain / 1e3),
                           "what": "one PIV call per pair on device-resident images, same kernels",
                           "e2e_value": info["total_ia"] / min(plain_e2e),
                           "e2e_what": "one PIV call per pair from host numpy arrays (best of 2 runs)"},
            "speedup_vs_plain": ms_plain / ms,
            "e2e": {"value": info["total_ia"] * len(e2e) / sum(e2e), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": info["launches"] * args.steps,
            "roofline": {"bound": "fp32", "achieved": flops / (ms / 1e3) / 1e12, "peak": fp32_peak / 1e12,
                         "unit": "TFLOP/s", "frac": flops / (ms / 1e3) / fp32_peak, "traffic": None,
                         "algorithmic_flop_per_step": flops,
                         "peak_source": f"148 SM x 128 FP32 lanes x 2 x sm_max_mhz ({src})"},
            "cpu_baseline": None, "clocks": clk.summary()}
    plan.close()
    return line


# ---------------------------------------------------------------------------
# the serving workload: Poisson arrivals of 2D+t and 3D+t requests
# ---------------------------------------------------------------------------
def run_serve(args):
    rank, _, world = dist_env()
    if rank != 0:  # a single-GPU workload: under a multi-rank launch rank 0 runs it alone
        return None
    from multi_quickpiv_b200 import setPIVParameters, synth
    from multi_quickpiv_b200.serve import Server
    t0 = time.time()
    kinds = []
    # 2D+t: 2048^2 Float32, NSQECC IS 32 SM 16 step 8, 100 requests/s over 4 streams
    for k in range(4):
        tg = synth.TaylorGreenStream((2048, 2048), seed_stream=70 + k)
        kinds.append(("2d", [tg.next() for _ in range(6)],
                      setPIVParameters(corr_alg="nsqecc", interSize=32, searchMargin=16, step=8), 25.0))
    # 3D+t: 256^3 Float32, FFTCC IS 32 SM 16 step 16, 5 requests/s
    tg = synth.TaylorGreenStream((256, 256, 256), seed_stream=80)
    kinds.append(("3d", [tg.next() for _ in range(4)],
                  setPIVParameters(corr_alg="fft", interSize=32, searchMargin=16, step=16), 5.0))
    gen_s = time.time() - t0
    g = np.random.default_rng(2026)
    horizon = args.steps / 105.0  # seconds of arrivals for ~steps requests
    events = []
    for ki, (_, frames, _, rate) in enumerate(kinds):
        t = 0.0
        while True:
            t += g.exponential(1.0 / rate)
            if t > horizon:
                break
            events.append((t, ki))
    events.sort()
    srv = Server(slots=4)
    sids = [srv.open_stream(fr[0], p) for _, fr, p, _ in kinds]
    for ki, (_, fr, _, _) in enumerate(kinds):  # warm-up: one request per stream
        srv.result(srv.submit(sids[ki], fr[1]))
    srv.reset_stats()
    nxt = [2] * len(kinds)
    rids = []
    with ClockSampler(0) as clk:
        ts = time.perf_counter()
        for ta, ki in events:
            while time.perf_counter() - ts < ta:
                pass
            fr = kinds[ki][1]
            rids.append((ki, srv.submit(sids[ki], fr[nxt[ki] % len(fr)])))
            nxt[ki] += 1
        lat = {"2d": [], "3d": []}
        for ki, rid in rids:
            lat[kinds[ki][0]].append(srv.result(rid)[2])
    st = srv.stats()
    srv.close()
    # plain per-request path: PIV() from host arrays, one request at a time, same arrivals
    import multi_quickpiv_b200 as mq
    plain = {"2d": [], "3d": []}
    ts = time.perf_counter()
    busy_until = 0.0
    for ta, ki in events:
        now = time.perf_counter() - ts
        if now < ta:
            time.sleep(ta - now)
        fr, p = kinds[ki][1], kinds[ki][2]
        mq.PIV(fr[0], fr[1], p)
        plain[kinds[ki][0]].append((time.perf_counter() - ts - ta) * 1e3)

    def pct(v, q):
        return float(np.percentile(v, q)) if len(v) else None
    ia2 = ((2048 - 32) // 8 + 1) ** 2
    ia3 = ((256 - 32) // 16 + 1) ** 3
    line = {"metric": METRIC, "value": st["ia_per_s"], "unit": UNIT, "n_gpus": 1, "steps": len(events),
            "warmup": len(kinds), "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (Taylor-Green advected particle streams)",
            "config": {"workload": "serving: Poisson arrivals, 2D+t 2048^2 NSQECC at 100/s (4 streams) and "
                                   "3D+t 256^3 FFTCC at 5/s", "slots": 4, "frames_generation_s": gen_s,
                       "ia_per_request": {"2d": ia2, "3d": ia3}},
            "latency_ms": {"p50": st["p50_ms"], "p99": st["p99_ms"], "max": st["max_ms"],
                           "2d_p50": pct(lat["2d"], 50), "2d_p99": pct(lat["2d"], 99),
                           "3d_p50": pct(lat["3d"], 50), "3d_p99": pct(lat["3d"], 99),
                           "queued_p50": st["wait_p50_ms"], "queued_p99": st["wait_p99_ms"],
                           "running_p50": st["run_p50_ms"], "running_p99": st["run_p99_ms"]},
            "admitted_while_busy": st["admitted_while_busy"], "completed": st["completed"], "failed": st["failed"],
            "plain_path_latency_ms": {"2d_p50": pct(plain["2d"], 50), "2d_p99": pct(plain["2d"], 99),
                                      "3d_p50": pct(plain["3d"], 50), "3d_p99": pct(plain["3d"], 99),
                                      "what": "PIV() per request from host arrays, one at a time, same arrivals"},
            "e2e": {"value": st["ia_per_s"], "unit": UNIT,
                    "h2d_bytes_per_step": int(2048 * 2048 * 4), "d2h_bytes_per_step": int(ia2 * 2 * 8)},
            "gpu_launches": None, "roofline": None, "cpu_baseline": None, "clocks": clk.summary()}
    return line


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--alg", default="nsqecc", choices=["nsqecc", "zncc", "fft"])
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-budget", type=float, default=10.0)
    ap.add_argument("--workload", default="vortex2048", choices=["vortex2048", "shear3d", "batch64", "serve", "window256"],
                    help="vortex2048: 2D vortex pair (--size, --alg); window256: the same pair at interSize 128, "
                         "margin 64, step 32 (search windows of 256); shear3d: 512x512x256 FFTCC volumes; "
                         "batch64: 64 mixed pairs with 3-pass refinement (batch plans vs per-pair calls); "
                         "serve: Poisson request streams (latency p50/p99; --steps = requests)")
    ap.add_argument("--chunk3d", type=int, default=0, help="IAs per 3D chunk (0: autotuned in warm-up)")
    ap.add_argument("--plan-only", action="store_true",
                    help="batch64: time the plan alone (default options), e.g. for a launch list")
    ap.add_argument("--no-extras", action="store_true",
                    help="vortex2048: skip the batch64, serve and shear3d summaries added to the line")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch64":
        line = run_batch(args)
    elif args.workload == "serve":
        line = run_serve(args)
    else:
        line = run_ours(args)
        if line is not None and args.workload == "vortex2048" and line["n_gpus"] == 1 and not args.no_extras:
            line["extras"] = extras(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def extras(args):
    """The other configured workloads, measured in the same run and summarised
    beside the headline line: the 512x512x256 3D FFTCC pass, the 64-pair
    batch (plan vs one PIV call per pair) and serving (p50/p99 latency vs the
    plain per-request path).  Each runs with its own reduced step count; a
    failure is reported in its entry and never fails the line."""
    import copy

    import torch
    out = {}
    jobs = [("shear3d", lambda a: run_ours(a), dict(workload="shear3d", steps=max(5, args.steps // 4), warmup=3,
                                                    no_cpu=True, chunk3d=0)),
            ("batch64", lambda a: run_batch(a), dict(workload="batch64", steps=max(4, args.steps // 5), warmup=3)),
            ("serve", lambda a: run_serve(a), dict(workload="serve", steps=max(200, args.steps)))]
    for name, fn, over in jobs:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.time()
        try:
            ln = fn(a)
            keep = ("value", "ms_per_step", "steps", "e2e", "config", "speedup_vs_plain", "plain_path",
                    "latency_ms", "plain_path_latency_ms", "admitted_while_busy", "completed", "failed",
                    "gpu_launches", "clocks")
            ent = {k: ln[k] for k in keep if k in ln}
            if ln.get("roofline"):
                ent["roofline"] = {k: ln["roofline"][k] for k in ("achieved", "peak", "unit", "frac", "kernel_ms")
                                   if k in ln["roofline"]}
        except Exception as e:  # reported, never fatal
            ent = {"error": f"{type(e).__name__}: {e}"}
        ent["wall_s"] = time.time() - t0
        out[name] = ent
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    sys.exit(main())
