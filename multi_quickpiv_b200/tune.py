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
