"""Autotuner for the grouped traversal's launch shape (no reference counterpart).

Three knobs: bodies per lane (buckets of up to 32 or 64 bodies), warps per
block (2, 4 or 8) and, with the reference opening test, the super-bucket size
of the two-level walk (0 = single level).  `tune(engine)` times every shape on the engine's current
tree with CUDA events and keeps the fastest; results are remembered per
(GPU, opening test, theta, size class) in a JSON file next to this module so
a later run on the same kind of GPU and workload can reuse them.
"""
from __future__ import annotations

import json
import math
import os

import torch

SHAPES = ((1, 2), (1, 4), (1, 8), (2, 2), (2, 4), (2, 8))
SUPERS = (0, 512, 1024)
CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tuned.json")


def _key(engine):
    name = torch.cuda.get_device_name(engine.state.device).replace(" ", "_")
    return f"{name}|mac{engine.mac}|theta{engine.config.THETA:.3f}|log2n{int(round(math.log2(max(engine.state.n, 1))))}"


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _apply(engine, bpl, warps, super_bodies=0):
    engine.bodies_per_lane = bpl
    engine.block_warps = warps
    engine.tree_manager.rebucket(32 * bpl)
    engine.set_super_bodies(super_bodies)


def tune(engine, shapes=SHAPES, supers=SUPERS, reps=3, use_cache=True, save=True):
    """Pick the fastest (bodies_per_lane, block_warps, super-bucket size) for
    `engine` (grouped mode, tree already built by forces_only/step).  Returns
    a report dict."""
    key = _key(engine)
    if engine.mac not in (0, 3):   # the two-level walk exists for the reference test only
        supers = (0,)
    cache = _load() if use_cache else {}
    if key in cache and len(cache[key].get("shape", [])) == 3:
        _apply(engine, *cache[key]["shape"])
        return dict(cache[key], cached=True)
    times = {}
    configs = [(bpl, warps, sb) for bpl, warps in shapes for sb in supers]
    for bpl, warps, sb in configs:
        _apply(engine, bpl, warps, sb)
        engine.compute_forces()              # warm-up of this shape
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            engine.compute_forces()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        times[f"{bpl}x{warps}s{sb}"] = best
    bpl, warps, sb = min(configs, key=lambda c: times[f"{c[0]}x{c[1]}s{c[2]}"])
    _apply(engine, bpl, warps, sb)
    report = {"shape": [bpl, warps, sb], "ms": times}
    if save:
        cache = _load()
        cache[key] = report
        try:
            with open(CACHE, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return dict(report, cached=False)
