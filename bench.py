"""Benchmark of the PIV hot path: interrogation-area (IA) correlations/s.

Workload (default): the 2048x2048 Float32 Lamb-Oseen vortex pair with ramp and
gain, interSize 32, searchMargin 16, step 8 (64,009 IAs per pair), NSQECC
(the reference's default algorithm; --alg zncc for ZNCC).  One step = one PIV
of one image pair.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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


def flops_per_ia(cs=64, P=33, IS=32, norm=True):
    """Reference-equivalent FLOPs of one 2D IA correlation (unpruned r2c/c2r of
    size cs^2, conj-multiply, peak scan; +normalisation for ZNCC/NSQECC)."""
    Nc = cs * cs
    B = (cs // 2 + 1) * cs
    f = 3 * 2.5 * Nc * math.log2(Nc) + 6 * B + P * P
    if norm:
        f += 12 * P * P + 2 * IS * IS
    return f


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
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

    def summary(self):
        if self.proc is None or self.out is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def make_workload(args):
    from multi_quickpiv_b200 import synth
    i1, i2, _ = synth.pair_2d_vortex(shape=(args.size, args.size))
    return i1, i2


def params_for(args):
    from multi_quickpiv_b200 import setPIVParameters
    return setPIVParameters(corr_alg=args.alg, interSize=(32, 32), searchMargin=(16, 16), step=(8, 8),
                            computeSN=False)


# ---------------------------------------------------------------------------
def cpu_baseline_sample(i1, i2, args, budget_s=12.0):
    """The oracle restatement timed on this host on a bounded sample of the
    workload's IAs; returns IA/s, threads used and the sample description."""
    import oracle.cpu_ref as cref
    if cref.available():
        return cref.time_sample(i1, i2, args.alg, budget_s=budget_s)
    import oracle.piv_oracle as O
    p = O.set_piv_parameters(corr_alg=args.alg, interSize=(32, 32), searchMargin=(16, 16), step=(8, 8))
    p.ndims = 2
    sub1, sub2 = i1[:288, :288].astype(np.float64), i2[:288, :288].astype(np.float64)
    t0 = time.perf_counter()
    VF, _ = O.piv_single_pass(sub1, sub2, p)
    dt = time.perf_counter() - t0
    n = VF.shape[1] * VF.shape[2]
    return {"value": n / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"NumPy Float64 oracle, {n} IAs of a 288x288 crop, {dt:.1f} s"}


def run_reference(args):
    rank, local, world = dist_env()
    if rank != 0:
        return 0
    i1, i2 = make_workload(args)
    import oracle.cpu_ref as cref
    if not cref.available():
        cref.build()
    K, W = args.steps, args.warmup
    res = None
    times = []
    for it in range(W + K):
        r = cref.time_sample(i1, i2, args.alg, budget_s=args.ref_budget)
        if it >= W:
            times.append(r)
        res = r
    vals = [r["value"] for r in times]
    value = statistics.mean(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": 1e3 * args.n_ia_full / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"vortex pair {args.size}x{args.size} float32, {args.alg}, IS 32 SM 16 step 8",
                       "n_ia_per_pair": args.n_ia_full},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": res["cores"], "kind": res["kind"],
                             "sample": res["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    rank, local, world = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import multi_quickpiv_b200 as mq
    from multi_quickpiv_b200 import _lib
    ctx = _lib.Context(local)
    i1, i2 = make_workload(args)
    params = params_for(args)
    params.ndims = 2
    H, Wd = i1.shape
    vf = mq.get_vectorfield_size(i1.shape, params)
    n_ia = vf[0] * vf[1]

    # device-resident inputs (column-major, Julia order)
    d1 = mq.piv._colmajor_torch(torch.from_numpy(i1).to(dev))
    d2 = mq.piv._colmajor_torch(torch.from_numpy(i2).to(dev))
    VF = torch.zeros((vf[1], vf[0], 2), dtype=torch.float64, device=dev)
    cp = params.to_c()
    import ctypes as C
    dims = (C.c_int64 * 3)(H, Wd, 1)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def step():
        rc = ctx.lib.mqp_piv_device(ctx.handle, C.c_void_p(d1.data_ptr()), C.c_void_p(d2.data_ptr()), None, None,
                                    _lib.MQP_F32, 2, dims, C.byref(cp), C.c_void_p(VF.data_ptr()), None,
                                    C.c_void_p(stream.cuda_stream))
        _lib.check(rc, ctx.handle)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ctx.profile_enable(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))  # evict the inputs from L2 between steps (not timed)
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    prof = ctx.profile_read()
    ctx.profile_enable(False)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * n_ia * args.steps / (total_ms / 1e3)

    # ---- e2e through the public API from pinned host memory ----
    h1p = torch.empty(H * Wd, dtype=torch.float32, pin_memory=True).numpy().reshape((H, Wd), order="F")
    h2p = torch.empty(H * Wd, dtype=torch.float32, pin_memory=True).numpy().reshape((H, Wd), order="F")
    h1p[...] = i1
    h2p[...] = i2
    for _ in range(max(1, args.warmup // 2)):
        mq.PIV(h1p, h2p, params, context=ctx)
    e2e_t = []
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        VFh, _ = mq.PIV(h1p, h2p, params, context=ctx)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_t)
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * n_ia * args.steps / e2e_s

    peaks, src = measured_peaks()
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6
    kern_ms = prof["ms_piv"] / max(prof["launches_piv"], 1)
    fl = flops_per_ia(norm=args.alg != "fft") * n_ia
    achieved = fl / (kern_ms / 1e3)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "piv2d_traffic.json")) as f:
            tr = json.load(f)
        # measured DRAM bytes of one launch, scaled by interrogation areas
        traffic = tr["dram_bytes_per_launch"] * n_ia / tr["ia_per_launch"]
    except Exception:
        pass
    roof = {"bound": "fp32", "kernel": "piv2d_kernel", "achieved": achieved / 1e12, "peak": fp32_peak / 1e12,
            "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
            "traffic_unit": "bytes per launch (ncu dram__bytes_read+write, profiles/piv2d_traffic.json)",
            "algorithmic_bytes_per_launch": 2 * H * Wd * 4 + (H + 1) * (Wd + 1) * 8 + n_ia * 16,
            "peak_source": f"148 SM x 128 FP32 lanes x 2 x sm_max_mhz from MEASURED_PEAKS.json ({src})",
            "kernel_ms": kern_ms, "algorithmic_flop_per_ia": flops_per_ia(norm=args.alg != "fft"),
            "hbm_frac_of_measured": (2 * H * Wd * 4 + n_ia * 16) / (kern_ms / 1e3) / (peaks.get("hbm_gbs", 6650) * 1e9)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline_sample(i1, i2, args)
        except Exception as e:  # reported, never fatal
            cpu = {"value": None, "error": str(e)}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"vortex pair {args.size}x{args.size} float32, {args.alg}, IS 32 SM 16 step 8",
                           "n_ia_per_pair": n_ia, "parallelism": f"replicas x{world}",
                           "l2": "flushed between steps by a 256 MiB write outside the timed events",
                           "compute": "FP32 FFTs, FP64 integral images and normalisation"},
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": int(2 * H * Wd * 4),
                        "d2h_bytes_per_step": int(n_ia * 2 * 8)},
                "gpu_launches": int(prof["launches_piv"] + prof["launches_integral"] * (2 if args.alg != "fft" else 0)
                                    + (2 * prof["launches_integral"] if args.alg == "zncc" else 0)),
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
                "kernel_ms": {"piv2d": kern_ms, "integral_scans": prof["ms_integral"] / max(args.steps, 1)}}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


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
    args = ap.parse_args(argv)
    args.n_ia_full = ((args.size - 32) // 8 + 1) ** 2
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
