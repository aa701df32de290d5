"""Autotuner for the persistent enumeration kernels.

Picks, by timing the real kernel on the real input (CUDA events on the launch
stream, device-resident inputs), the launch and schedule parameters that the
results never depend on:
  * split granularity   heavy-root tasks aim at total / (g x warps) cost
  * warps per CTA       4 or 8 (the persistent grid keeps 32 warps per SM)
  * queue chunk         tasks taken per atomic on the device queue
  * intersection path   clique plans: bitmap (0) or generic plan interpreter (1)
  * register budget     GMatch kernel built for 4 or 6 CTAs of 256 threads per SM
  * MCE hand-off        check interval of walks for idle warps (bench's MCE space)
Coordinate descent over that grid, one parameter at a time, starting from the
library defaults and repeated until a full pass changes nothing (parameters
interact: whether splitting pays depends on the register budget, for one);
every candidate is run `reps` times and its best time kept.
"""
from __future__ import annotations

import itertools


def _time(torch, stream, fn, reps):
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune(run, base: dict, space: dict, reps: int = 2, max_passes: int = 3):
    """run(**opts) enqueues one enumeration on the current torch stream.
    Returns (best opts, best ms, log of (opts, ms))."""
    import torch
    stream = torch.cuda.current_stream()
    cur = dict(base)
    run(**cur)  # warm-up (module load, buffers)
    torch.cuda.synchronize()
    best_ms = _time(torch, stream, lambda: run(**cur), reps)
    log = [(dict(cur), best_ms)]
    seen = {tuple(sorted(cur.items()))}
    for _ in range(max_passes):
        changed = False
        for key, values in space.items():
            for v in values:
                cand = dict(cur, **{key: v})
                sig = tuple(sorted(cand.items()))
                if sig in seen:
                    continue
                seen.add(sig)
                ms = _time(torch, stream, lambda: run(**cand), reps)
                log.append((cand, ms))
                if ms < best_ms:
                    best_ms, cur, changed = ms, cand, True
        if not changed:
            break
    return cur, best_ms, log


DEFAULT_SPACE = {
    "ctas_per_sm": [4, 6],
    "granularity": [4, 16, 64],
    "warps_per_block": [4, 8],
    "chunk": [1, 4, 16],
}


def grid(space):
    keys = list(space)
    for vals in itertools.product(*(space[k] for k in keys)):
        yield dict(zip(keys, vals))
