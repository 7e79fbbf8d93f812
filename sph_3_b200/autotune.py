"""Project-written autotuner for the walk launch parameters.

Tunables (all runtime, no recompilation):
  leaf_size   octree leaf capacity (smaller leaves: tighter candidate sets,
              deeper trees and more nodes to walk)
  walk_warps  warps per walk block (one warp walks one group of <= 32
              particles; the block width trades shared-memory footprint per
              block against scheduling granularity)
  stack_cap   walk-stack entries per warp (wider pops need more room; the
              capacity must stay >= 7 (max_level + 2) + 32)

Each candidate is timed on the caller's own particle set: a few full KDK
steps (CUDA graph, CUDA events on a private stream) after warm-up.  The best
configuration is cached as JSON, keyed by GPU name, particle-count bucket,
number of systems, precision and boundary type, so later runs of the same
workload shape start from it.  The cache lives in $SPH3_AUTOTUNE_CACHE or
~/.cache/sph3_b200/autotune.json.
"""
from __future__ import annotations

import itertools
import json
import math
import os
from typing import Dict, Iterable, Optional, Tuple

DEFAULT_GRID = {
    "leaf_size": (8, 12, 16, 24, 32),
    "walk_warps": (2, 4, 8),
    "stack_cap": (768, 1024, 2048),
}


def cache_path() -> str:
    p = os.environ.get("SPH3_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "sph3_b200", "autotune.json")


def workload_key(gpu_name: str, n: int, ncloud: int, precision: str, periodic: bool) -> str:
    bucket = int(round(math.log2(max(n, 1))))
    cb = int(round(math.log2(max(ncloud, 1))))
    return "%s|n2^%d|clouds2^%d|%s|%s" % (gpu_name, bucket, cb, precision, "periodic" if periodic else "open")


def load_cache(path: Optional[str] = None) -> Dict[str, dict]:
    path = path or cache_path()
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(data: Dict[str, dict], path: Optional[str] = None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp%d" % os.getpid()
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(grid: Dict[str, Iterable], max_level: int) -> Iterable[dict]:
    keys = sorted(grid)
    for combo in itertools.product(*(grid[k] for k in keys)):
        c = dict(zip(keys, combo))
        if "stack_cap" in c and c["stack_cap"] < 7 * (max_level + 2) + 32:
            continue
        yield c


def _time_steps(ctx, dt: float, steps: int, warmup: int) -> float:
    import torch
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ctx.step(dt, warmup, stream=s.cuda_stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.step(dt, steps, stream=s.cuda_stream)
        e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def autotune(ctx, dt: float = 1e-3, steps: int = 3, warmup: int = 4, grid: Optional[dict] = None,
             use_cache: bool = True, restore_state: bool = True) -> Tuple[dict, Dict[str, float]]:
    """Times every candidate on ctx's particles, applies the fastest and
    returns (best parameters, {candidate: ms per step}).  The particle state
    is saved before and restored after, so tuning does not advance the run."""
    import torch
    grid = grid or DEFAULT_GRID
    name = torch.cuda.get_device_name()
    cfg0 = ctx.config
    key = workload_key(name, ctx.n, getattr(ctx, "ncloud", 1), cfg0.precision,
                       any(b > 0 for b in cfg0.box))
    if use_cache:
        hit = load_cache().get(key)
        if hit:
            ctx.set_config(cfg0.replace(**hit["best"]))
            return hit["best"], hit.get("times", {})
    saved = None
    if restore_state:
        saved = {f: ctx.get_field(f) for f in ("pos", "vel", "u", "u_prev", "h", "acc", "dudt_prev")}
    times = {}
    best, best_ms = None, float("inf")
    for cand in candidates(grid, cfg0.max_level):
        ctx.set_config(cfg0.replace(**cand))
        ms = _time_steps(ctx, dt, steps, warmup)
        times[json.dumps(cand, sort_keys=True)] = ms
        if ms < best_ms:
            best, best_ms = cand, ms
        if saved is not None:
            for f, v in saved.items():
                ctx.set_field(f, v)
    ctx.set_config(cfg0.replace(**best))
    if use_cache:
        data = load_cache()
        data[key] = {"best": best, "ms_per_step": best_ms, "times": times}
        save_cache(data)
    return best, times
