"""Launch-schedule autotuner of the tensor-core layer kernels.

The fused layer kernel's results do not depend on its schedule (pipeline
stages, tensor-memory accumulators, resident CTAs per SM:
``spk_set_conv_schedule``), its speed does, and the best choice depends on
the layer's shape (K blocks per tile, output channels, image size).  The
tuner times each candidate on the real call with CUDA events and keeps the
fastest; results are cached per shape key by the caller.
"""

from __future__ import annotations

import torch

from ._lib import SpykerError

# (stages, accumulators, CTAs per SM); 0 = the kernel's automatic choice
CANDIDATES = [(0, 0, 0), (2, 0, 0), (3, 0, 0), (6, 0, 0), (0, 1, 0), (3, 1, 0), (0, 0, 1), (0, 0, 2)]


def time_call(run, reps: int = 3) -> float:
    """Mean milliseconds of `run()` over `reps` calls after one warm-up."""
    run()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        run()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def best_schedule(run, reps: int = 3, candidates=CANDIDATES):
    """The fastest schedule for `run(schedule)`; candidates that the kernel
    rejects (for this shape) are skipped."""
    timings = {}
    for st in candidates:
        try:
            timings[st] = time_call(lambda: run(st), reps)
        except SpykerError:
            continue
    if not timings:
        return (0, 0, 0)
    best = min(timings, key=timings.get)
    best_schedule.last = timings
    return best
