"""Autotuner of the launch schedule (CTA size, CTAs per SM, drain kind, atomic mode,
eager sub-rounds, Delta multiplier) for a given graph and batch.

Coordinate descent over a small discrete space, timing each candidate with the
engine's own CUDA-event time (median of `reps` runs); results are cached in a
JSON file keyed by the graph's statistics and the batch size, so a workload is
tuned once. Every candidate computes the same distances and parents: the
schedule never changes results.
"""
from __future__ import annotations

import json
import os
import statistics
from dataclasses import asdict, replace
from pathlib import Path
from typing import Callable, Dict, Optional, Tuple

from .solver import AtomicMode, Compaction, GpuAlgo, GpuOptions, Mapping, Policy, Schedule

LAUNCH_SHAPES = [(256, 4), (512, 2), (1024, 1)]       # (threads per CTA, CTAs per SM)
# asynchronous drains: automatic (a window per instance where that applies), one shared
# window with CTA passes, warp workers
SCHEDULES = [Schedule.Auto, Schedule.Async, Schedule.Warp]
ATOMICS = [AtomicMode.MinRBA, AtomicMode.MinNoCheck]
EAGER = [0, 2, 4, 8]
DELTA_MULT = [0.25, 0.5, 1.0, 2.0, 4.0, 16.0]


def cache_path() -> Path:
    p = os.environ.get("PFG_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "pathfinding_gpu_b200" / "tune.json"


def signature(g, batch: int, algo: GpuAlgo) -> str:
    return (f"n{g.n}-m{g.m}-deg{g.avgDeg:.2f}-maxdeg{g.maxDeg}-w{g.avgW:.1f}-maxw{g.maxW}"
            f"-xy{int(g.hasCoords())}-k{batch}-{algo.name}")


def _load() -> Dict:
    p = cache_path()
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


def _store(key: str, opt: GpuOptions, ms: float) -> None:
    p = cache_path()
    d = _load()
    o = asdict(opt)
    o = {k: (int(v) if hasattr(v, "value") else v) for k, v in o.items()}
    d[key] = {"options": o, "ms": ms}
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(json.dumps(d, indent=1))
    except OSError:
        pass


def cached(key: str) -> Optional[GpuOptions]:
    e = _load().get(key)
    if not e:
        return None
    o = e["options"]
    return GpuOptions(algo=GpuAlgo(o["algo"]), mapping=Mapping(o["mapping"]), atomic=AtomicMode(o["atomic"]),
                      delta=o["delta"], blockSize=o["blockSize"], syncEvery=o["syncEvery"],
                      compaction=Compaction(o.get("compaction", 0)), policy=Policy(o.get("policy", 0)),
                      eager=o["eager"], blocksPerSM=o["blocksPerSM"], schedule=Schedule(o.get("schedule", 0)))


def tune(time_fn: Callable[[GpuOptions], float], base: GpuOptions, auto_delta: int, reps: int = 2,
         key: Optional[str] = None, use_cache: bool = True) -> Tuple[GpuOptions, float, list]:
    """Returns (best options, best ms, trial log). time_fn(opt) -> device ms of one run."""
    if key and use_cache:
        hit = cached(key)
        if hit is not None:
            return hit, float("nan"), []
    log = []

    def measure(o: GpuOptions) -> float:
        t = statistics.median(time_fn(o) for _ in range(reps))
        log.append((asdict(o), t))
        return t

    best = replace(base, mapping=Mapping.Hybrid)
    best_t = measure(best)
    knobs = []
    knobs.append([replace(best, blockSize=b, blocksPerSM=s) for b, s in LAUNCH_SHAPES])
    if base.algo == GpuAlgo.DeltaStep:
        knobs.append([replace(best, schedule=sc) for sc in SCHEDULES])
    knobs.append([replace(best, atomic=a) for a in ATOMICS])
    knobs.append([replace(best, eager=e) for e in EAGER])
    if base.algo == GpuAlgo.DeltaStep:
        knobs.append([replace(best, delta=max(1, int(round(auto_delta * f)))) for f in DELTA_MULT])
    names = ["blockSize"] + (["schedule"] if base.algo == GpuAlgo.DeltaStep else []) + ["atomic", "eager"] + \
        (["delta"] if base.algo == GpuAlgo.DeltaStep else [])
    for i, cands in enumerate(knobs):
        # rebuild the candidates on the current best (earlier knobs may have moved)
        field = {"blockSize": ("blockSize", "blocksPerSM"), "schedule": ("schedule",), "atomic": ("atomic",),
                 "eager": ("eager",), "delta": ("delta",)}[names[i]]
        for c in cands:
            trial = replace(best, **{f: getattr(c, f) for f in field})
            if trial == best:
                continue
            t = measure(trial)
            if t < best_t:
                best, best_t = trial, t
    if key:
        _store(key, best, best_t)
    return best, best_t, log
