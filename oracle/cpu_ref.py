"""Loader/timer for the oracle's C++/OpenMP restatement (oracle/cpu).

Test infrastructure and the CPU baseline of bench.py only.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu", "mqp_cpu.cpp")
LIB = os.path.join(HERE, "cpu", "_build", "libmqp_cpu.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def build(force=False) -> str:
    if not os.path.exists(SRC):
        return ""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["g++", "-O3", "-march=native", "-fopenmp", "-std=c++17", "-fPIC", "-shared",
           "-I", os.path.join(os.path.dirname(HERE), "include"), SRC, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        # a portable build for hosts whose gcc rejects -march=native
        cmd.remove("-march=native")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stdout + r.stderr)
    return LIB


def load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB)
    return _lib


DIAG_FIELDS = ("top1", "top2", "scale", "sn_den", "skipped")


def piv(img1, img2, cparams, mask=None, mask_skip=None, nthreads=0, ia_begin=0, ia_end=-1, diag=False):
    """Run the C++ restatement; cparams is a multi_quickpiv_b200._lib.MqpParams
    (the same POD the C ABI takes).  Returns (VF, SN) shaped like PIV's, plus,
    with diag=True, a dict of per-IA arrays (vector-field shape) describing the
    similarity block on the lags first_fullovp_peak searches: the largest and
    second-largest values, the largest magnitude, compute_SN's denominator and
    a skipped flag."""
    lib = load()
    a1 = np.asarray(img1)
    dt = np.float64 if a1.dtype == np.float64 else np.float32
    f1 = np.asfortranarray(a1, dtype=dt)
    f2 = np.asfortranarray(np.asarray(img2), dtype=dt)
    fm = np.asfortranarray(np.asarray(mask), dtype=dt) if mask is not None else None
    fs = np.asfortranarray(np.asarray(mask_skip), dtype=dt) if mask_skip is not None else None
    N = a1.ndim
    dims = (C.c_int64 * 3)(*(list(a1.shape) + [1] * (3 - N)))
    vf = []
    for d in range(N):
        st = cparams.step[d] if cparams.has_step else cparams.interSize[d] - cparams.overlap[d]
        stop = a1.shape[d] - cparams.interSize[d] + 1
        vf.append(0 if stop < 1 else (stop - 1) // st + 1)
    VF = np.zeros((N,) + tuple(vf), dtype=np.float64, order="F")
    SN = np.zeros(tuple(vf), dtype=np.float64, order="F")
    ptr = lambda x: None if x is None else x.ctypes.data_as(C.c_void_p)
    args = [ptr(f1), ptr(f2), ptr(fm), ptr(fs), C.c_int(1 if dt == np.float64 else 0), C.c_int(N), dims,
            C.byref(cparams), ptr(VF), ptr(SN), C.c_int(nthreads), C.c_int64(ia_begin), C.c_int64(ia_end)]
    D = None
    if diag:
        D = np.zeros((len(DIAG_FIELDS),) + tuple(vf), dtype=np.float64, order="F")
        fn = lib.mqp_cpu_piv_diag
        args.append(ptr(D))
    else:
        fn = lib.mqp_cpu_piv
    fn.restype = C.c_int
    rc = fn(*args)
    if rc != 0:
        raise RuntimeError(f"mqp_cpu_piv failed: {rc}")
    out = (VF, (SN if cparams.computeSN else None))
    if diag:
        out = out + ({k: D[i] for i, k in enumerate(DIAG_FIELDS)},)
    return out


def threads() -> int:
    fn = load().mqp_cpu_max_threads
    fn.restype = C.c_int
    return int(fn())


def time_sample(i1, i2, alg, budget_s=12.0, IS=32, SM=16, step=8):
    """IA/s of the restatement on all host threads over a bounded prefix of
    the workload's IAs (column-major IA order), sized to ~budget_s."""
    from multi_quickpiv_b200 import setPIVParameters
    nd = i1.ndim
    p = setPIVParameters(corr_alg=alg, interSize=(IS,) * nd, searchMargin=(SM,) * nd, step=(step,) * nd)
    p.ndims = nd
    cp = p.to_c()
    nth = threads()
    n_total = 1
    for d in range(i1.ndim):
        n_total *= (i1.shape[d] - IS) // step + 1
    n = min(n_total, (64 if nd == 2 else 2) * nth)
    t0 = time.perf_counter()
    piv(i1, i2, cp, nthreads=nth, ia_begin=0, ia_end=n)
    dt = time.perf_counter() - t0
    rate = n / max(dt, 1e-9)
    n2 = int(min(n_total, max(n, rate * budget_s)))
    t0 = time.perf_counter()
    piv(i1, i2, cp, nthreads=nth, ia_begin=0, ia_end=n2)
    dt2 = time.perf_counter() - t0
    return {"value": n2 / dt2, "unit": "IA/s", "cores": nth, "kind": "port",
            "sample": f"C++/OpenMP Float64 restatement, first {n2} of {n_total} IAs "
                      f"({i1.shape[0]}x{i1.shape[1]}{'x%d' % i1.shape[2] if i1.ndim == 3 else ''}, {alg}), "
                      f"{dt2:.1f} s on {nth} threads"}
