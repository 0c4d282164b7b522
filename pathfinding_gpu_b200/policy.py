"""Learned Delta policy: trace collection, training and inference (GPU kernels in pfg_policy.cu).

At every decision point of Delta-stepping (the first bucket and every bucket
advance) the persistent kernel computes 12 features of the frontier: the size of
the next bucket's input, the last bucket's items, arcs scanned and work ratio, and
from a sample of up to 64 frontier items their degree histogram (<= 4, 5-32, > 32
slots), the fraction of light arcs at the current Delta and the spread of their
tentative distances, plus the gap to the next key, Delta / avgW and the bucket
count (decision_features / frontier_sample in pfg_persistent.cuh); with the policy loaded it
evaluates a 12 -> 64 -> 64 -> 64 -> 16 MLP whose argmax c picks how the next
bucket runs: Delta = MULTIPLIERS[c % 8] x the automatic Delta, drained
asynchronously (c < 8) or in relaxation rounds (c >= 8). The policy changes the
schedule only; distances and parents are identical to the fixed-Delta run.

Training data comes from the solver itself: for each (graph, source) of the
synthetic families, fixed-Delta runs of every class (schedule x multiplier) are
timed and traced; every trace row of a graph gets the same soft target, a
softmax of the negative relative run times, so the network learns which class
wins from what the frontier and the graph look like.
"""
from __future__ import annotations

import ctypes as C
import statistics
from pathlib import Path
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .solver import GpuOptions, GpuSolver, Policy, Schedule

IN, H, OUT = 12, 64, 16
TRACE_W = 16
MULTIPLIERS = [0.0625, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0, 8.0]
# class c -> (schedule, multiplier); the kernel decodes c the same way
CLASSES = [(Schedule.Async, m) for m in MULTIPLIERS] + [(Schedule.Rounds, m) for m in MULTIPLIERS]


def class_name(c: int) -> str:
    sch, m = CLASSES[c]
    return f"{sch.name.lower()}x{m:g}"
SIZES = [("w1", (H, IN)), ("b1", (H,)), ("w2", (H, H)), ("b2", (H,)), ("w3", (H, H)), ("b3", (H,)),
         ("w4", (OUT, H)), ("b4", (OUT,)), ("in_mean", (IN,)), ("in_scale", (IN,))]
NP = sum(int(np.prod(s)) for _, s in SIZES)
WEIGHTS = Path(__file__).resolve().parent / "policy_weights.npz"


def init_params(seed: int = 0, mean=None, scale=None) -> np.ndarray:
    """He-initialised parameter image with the given input normalisation."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SIZES:
        if name.startswith("w"):
            parts.append(rng.normal(0, np.sqrt(2.0 / shape[1]), shape))
        elif name == "in_mean":
            parts.append(np.zeros(IN) if mean is None else np.asarray(mean))
        elif name == "in_scale":
            parts.append(np.ones(IN) if scale is None else np.asarray(scale))
        else:
            parts.append(np.zeros(shape))
    flat = np.concatenate([np.asarray(p, np.float64).reshape(-1) for p in parts]).astype(np.float32)
    assert flat.size == NP
    return flat


def normalisation(X: np.ndarray):
    mean = X.mean(axis=0)
    std = X.std(axis=0)
    return mean, 1.0 / np.where(std > 1e-6, std, 1.0)


def soft_targets(times_ms: Sequence[float], temperature: float = 0.05) -> np.ndarray:
    t = np.asarray(times_ms, np.float64)
    r = t / t.min() - 1.0
    e = np.exp(-r / temperature)
    return (e / e.sum()).astype(np.float32)


def grad(params, X, Y):
    lib = N.load()
    params = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    Y = np.ascontiguousarray(Y, np.float32)
    g = np.empty(NP, np.float32)
    loss = C.c_float()
    N.check(lib.pfg_policy_grad(N.ptr(params, N.f32), N.ptr(X, N.f32), N.ptr(Y, N.f32), len(X),
                                N.ptr(g, N.f32), C.byref(loss)))
    return float(loss.value), g


def train(X, Y, steps: int = 1500, lr: float = 3e-3, seed: int = 0,
          params: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Full-batch Adam on the GPU; returns (params, per-step loss)."""
    lib = N.load()
    X = np.ascontiguousarray(X, np.float32)
    Y = np.ascontiguousarray(Y, np.float32)
    if params is None:
        mean, scale = normalisation(X)
        params = init_params(seed, mean, scale)
    params = np.ascontiguousarray(params, np.float32).copy()
    losses = np.empty(steps, np.float32)
    N.check(lib.pfg_policy_train(N.ptr(params, N.f32), N.ptr(X, N.f32), N.ptr(Y, N.f32), len(X), steps,
                                 float(lr), N.ptr(losses, N.f32)))
    return params, losses


def infer(params, X) -> np.ndarray:
    lib = N.load()
    params = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    out = np.empty(len(X), np.uint32)
    N.check(lib.pfg_policy_infer(N.ptr(params, N.f32), N.ptr(X, N.f32), len(X), N.ptr(out, N.u32)))
    return out


def _sources(src) -> List[int]:
    """One source, or a batch of sources run as one multi-source launch."""
    return [int(src)] if isinstance(src, (int, np.integer)) else [int(x) for x in src]


def run_traced(solver: GpuSolver, src, opt: GpuOptions, cap: int = 4096):
    """One traced Delta-stepping run of one source or a batch: (stats, ms, trace rows [r, 16])."""
    lib = N.load()
    from .solver import GpuStats
    srcs = np.ascontiguousarray(_sources(src), np.uint32)
    c = opt.to_c()
    st = N.PfgStats()
    buf = np.empty((cap, TRACE_W), np.float32)
    rows = C.c_uint32()
    ms = C.c_float()
    N.check(lib.pfg_run_traced(solver.handle, N.ptr(srcs, N.u32), len(srcs), C.byref(c), C.byref(st),
                               N.ptr(buf, N.f32), cap, C.byref(rows), C.byref(ms)))
    return GpuStats.from_c(st), float(ms.value), buf[: rows.value].copy()


def collect(solver: GpuSolver, sources: Iterable[int], reps: int = 3, rows_per_run: int = 96,
            base: Optional[GpuOptions] = None, seed: int = 0):
    """Traces and soft targets from fixed-Delta sweeps over CLASSES (each element of
    `sources` is one source or a batch of sources run as one multi-source launch).

    Each source's sweep is normalised by its fastest multiplier and the curves of
    all sources of the graph are averaged; every trace row of the graph gets the
    soft target of that mean curve (one label per graph family, so run-to-run
    noise of a single source does not flip the class)."""
    rng = np.random.default_rng(seed)
    base = base or GpuOptions()
    auto = solver.autoDelta()
    traces, curves, table = [], [], []
    for src in sources:
        times = []
        for sched, mult in CLASSES:
            d = max(1, int(auto * mult))  # the kernel truncates the same product
            o = GpuOptions(**{**base.__dict__, "delta": d, "policy": Policy.Fixed, "schedule": sched})
            solver.run_state(_sources(src), o, copy=False)  # warm
            ts = []
            tr = None
            for r in range(reps):
                st, ms, rows = run_traced(solver, src, o)
                ts.append(ms)
                tr = rows
            times.append(statistics.median(ts))
            if len(tr) > rows_per_run:
                tr = tr[np.sort(rng.choice(len(tr), rows_per_run, replace=False))]
            traces.append(tr)
        curves.append(np.asarray(times) / min(times))
        srcs = _sources(src)
        table.append({"src": srcs[0] if len(srcs) == 1 else f"batch of {len(srcs)} from {srcs[0]}",
                      "times_ms": [round(t, 4) for t in times],
                      "best": class_name(int(np.argmin(times)))})
    mean_curve = np.mean(curves, axis=0)
    y = soft_targets(mean_curve)
    X = np.concatenate([tr[:, :IN] for tr in traces])
    Y = np.repeat(y[None, :], len(X), axis=0)
    return X, Y, table, [round(float(c), 4) for c in mean_curve]


def save(params: np.ndarray, path: Path = WEIGHTS, meta: Optional[dict] = None) -> None:
    np.savez(path, params=np.asarray(params, np.float32), meta=np.asarray(str(meta or {})))


def load(path: Path = WEIGHTS) -> np.ndarray:
    d = np.load(path)
    return d["params"].astype(np.float32)
