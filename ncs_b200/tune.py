"""Launch-configuration autotuner for the persistent solver.

The kernels pull tiles from a device-side queue, so the work per CTA adapts
by itself; what a launch fixes is how many CTAs (four warps, one tile per
warp at a time) stay resident per SM and the L-BFGS history size m.  Both
change speed but not the result's accuracy (the stopping rule is the same),
so the tuner times every candidate on the caller's own workload with CUDA
events and keeps the fastest.  Results are cached per workload key in
memory and, optionally, in a JSON file.

No counterpart in the reference, whose launch geometry is fixed
(cuda/pyCUDANCS/ncs.py:137-147: one 16-thread block per tile).
"""
import json
import os

import torch

DEFAULT_CANDIDATES = tuple({"ctas_per_sm": c, "m": m} for c in (2, 3, 4) for m in (1, 2, 4))

_cache = {}


def _time_ms(fn, warmup, reps):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def autotune(solver, run, key, candidates=DEFAULT_CANDIDATES, warmup=1, reps=2, path=None):
    """Time ``run()`` under each candidate (a dict of Solver parameters),
    leave ``solver`` set to the fastest and return (best, timings).

    ``run`` issues one solve on ``solver`` (e.g. a batched launch);
    ``key`` names the workload for the cache; ``path`` (optional) is a JSON
    file that keeps the choice across processes."""
    if path and os.path.exists(path) and key not in _cache:
        with open(path) as f:
            _cache.update(json.load(f))
    if key in _cache:
        best = _cache[key]["best"]
        solver.set_params(**best)
        return best, _cache[key]["ms"]
    timings = []
    for cand in candidates:
        solver.set_params(**cand)
        timings.append((_time_ms(run, warmup, reps), cand))
    ms, best = min(timings, key=lambda t: t[0])
    solver.set_params(**best)
    _cache[key] = {"best": best, "ms": [[t, c] for t, c in timings]}
    if path:
        with open(path, "w") as f:
            json.dump(_cache, f, indent=1)
    return best, _cache[key]["ms"]


def batch_key(solver):
    """Workload key of the batch registered on ``solver``: its tile count and
    stack count, rounded to the power of two above."""
    n = max(1, int(getattr(solver, "batch_tiles", 0)))
    s = max(1, len(getattr(solver, "_batch", []) or []))
    return "batch/t%d/s%d" % (1 << (n - 1).bit_length(), 1 << (s - 1).bit_length())
