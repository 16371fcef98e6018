"""Launch autotuning: picks launch parameters of the PIV path by timing them
on the caller's own workload.  Results never depend on the choice; only the
time does.

The tuned knobs are the ones the C ABI exposes through mqp_set_tuning
(include/mqp.h): the 3D chunk size (IAs per K3a/K3b/K3c round, which trades
scratch footprint and L2 reuse against launch count).
"""
from __future__ import annotations

from typing import Callable, Dict, Iterable, Tuple


def time_ms(fn: Callable[[], None], stream, reps: int = 2) -> float:
    """Mean device time of fn() on `stream` (a torch.cuda.Stream) over reps
    runs after one untimed run, by CUDA events on that stream."""
    import torch
    fn()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def autotune_chunk3d(ctx, step: Callable[[], None], stream,
                     candidates: Iterable[int] = (512, 1024, 2048, 4096),
                     reps: int = 2) -> Tuple[int, Dict[int, float]]:
    """Times `step` (one 3D PIV through ctx) for each chunk size, leaves ctx
    on the fastest and returns (chunk, {chunk: ms})."""
    res = {}
    for c in candidates:
        ctx.set_chunk3d(int(c), 0)
        res[int(c)] = time_ms(step, stream, reps)
    best = min(res, key=res.get)
    ctx.set_chunk3d(best, 0)
    return best, res


def autotune_batch(pairs, candidates=None, context=None, reps: int = 2):
    """Builds the batch plan of `pairs` with each candidate option set
    (dicts of mqp_batch_options fields), times one run of each by CUDA events
    and returns (best options, {str(options): ms}, the best plan)."""
    import torch

    from .batch import BatchPlan
    if candidates is None:
        candidates = [dict(grab=g, use_graph=1, chunk3d=c) for g in (1, 2, 4) for c in (0, 2048)]
    res = {}
    best = None
    for opt in candidates:
        plan = BatchPlan(pairs, opt, context)
        ms = time_ms(plan.run, torch.cuda.current_stream(plan.device), reps)
        res[str(opt)] = ms
        if best is None or ms < best[1]:
            if best is not None:
                best[2].close()
            best = (opt, ms, plan)
        else:
            plan.close()
    return best[0], res, best[2]
