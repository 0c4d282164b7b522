"""Trains the learned Delta policy on a GPU and writes pathfinding_gpu_b200/policy_weights.npz.

    python -m pathfinding_gpu_b200.train_policy [--out policy_weights.npz] [--report report.json]

1. Traces: for every (graph, source) of the training families (R-MAT scales 19-20
   with two edge factors and two weight ranges, seeds other than the evaluation
   graph's; grids of 256-768 per side; a road-like grid; batches of 32-64 sources on grids and
   the road-like grid, run as one multi-source launch), fixed-Delta
   runs of each class of policy.CLASSES (schedule x multiplier) are timed and
   traced.
2. Training: full-batch Adam with the hand-written kernels of pfg_policy.cu.
3. Evaluation on graphs NOT used for training (R-MAT scale 20, edge factor 16;
   the 1000 x 1000 grid): learned vs fixed automatic Delta, same sources, results
   compared word for word.
"""
from __future__ import annotations

import argparse
import json
import statistics
import sys
import time
from pathlib import Path

import numpy as np

from . import graphs as G
from . import policy as P
from .solver import GpuOptions, GpuSolver, Policy, unpack

TRAIN_FAMILIES = [
    ("rmat_s19_ef16_w255", lambda: G.rmat(19, 16, w_lo=1, w_hi=255, seed=16)),
    ("rmat_s19_ef8_w1000", lambda: G.rmat(19, 8, w_lo=1, w_hi=1000, seed=17)),
    ("rmat_s20_ef8_w255", lambda: G.rmat(20, 8, w_lo=1, w_hi=255, seed=18)),
    ("rmat_s20_ef16_w255_seed31", lambda: G.rmat(20, 16, w_lo=1, w_hi=255, seed=31)),
    ("rmat_s20_ef16_w255_seed32", lambda: G.rmat(20, 16, w_lo=1, w_hi=255, seed=32)),
    ("rmat_s20_ef16_w255_seed33", lambda: G.rmat(20, 16, w_lo=1, w_hi=255, seed=33)),
    ("grid_256", lambda: G.grid(256, 256, 21)),
    ("grid_512", lambda: G.grid(512, 512, 22)),
    ("grid_768", lambda: G.grid(768, 768, 23)),
    ("road_512", lambda: G.road(512, seed=24)),
    # batches of sources sharing one bucket sequence (multi-source launches)
    ("grid_512_k64", lambda: G.grid(512, 512, 25), 64),
    ("grid_768_k32", lambda: G.grid(768, 768, 26), 32),
    ("grid_768_k64", lambda: G.grid(768, 768, 27), 64),
    ("road_512_k64", lambda: G.road(512, seed=28), 64),
]
EVAL = [
    ("rmat_s20_ef16_seed2026", lambda: G.rmat(20, 16, seed=2026)),
    ("grid_1000_seed2026", lambda: G.grid(1000, 1000, 2026)),
    ("grid_1000_seed2026_k64", lambda: G.grid(1000, 1000, 2026), 64),
]


def timed(solver, src, opt, reps=5):
    srcs = P._sources(src)
    solver.run_state(srcs, opt, copy=False)
    return statistics.median(solver.run_state(srcs, opt, copy=False)[1] for _ in range(reps))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(P.WEIGHTS))
    ap.add_argument("--report", default=None)
    ap.add_argument("--sources", type=int, default=4)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=3e-3)
    args = ap.parse_args(argv)
    base = GpuOptions(blockSize=1024)
    report = {"families": {}, "eval": {}}
    Xs, Ys = [], []
    t0 = time.time()
    for fam in TRAIN_FAMILIES:
        name, make, k = fam if len(fam) == 3 else (*fam, 1)
        g = make()
        with GpuSolver(g, k) as s:
            if k == 1:
                srcs = G.pick_sources(g, args.sources, 7).tolist()
            else:  # two batches of k sources
                srcs = [tuple(G.uniform_vertices(g.n, k, 7 + b).tolist()) for b in range(2)]
            X, Y, table, curve = P.collect(s, srcs, base=base, reps=5)
        Xs.append(X)
        Ys.append(Y)
        report["families"][name] = {"n": g.n, "m": g.m, "rows": len(X), "sweeps": table, "mean_curve": curve}
        best = P.class_name(int(np.argmin(curve)))
        print(f"[traces] {name}: {len(X)} rows, best per source {[t['best'] for t in table]}, "
              f"family label {best}", flush=True)
    X = np.concatenate(Xs)
    Y = np.concatenate(Ys)
    params, losses = P.train(X, Y, steps=args.steps, lr=args.lr)
    acc = float(np.mean(P.infer(params, X) == np.argmax(Y, axis=1)))
    report["train"] = {"rows": len(X), "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                       "argmax_agreement": acc, "seconds": round(time.time() - t0, 1)}
    print(f"[train] rows {len(X)} loss {losses[0]:.4f} -> {losses[-1]:.4f}, argmax agreement {acc:.3f}", flush=True)
    P.save(params, Path(args.out), {"steps": args.steps, "lr": args.lr, "rows": len(X)})

    for fam in EVAL:
        name, make, k = fam if len(fam) == 3 else (*fam, 1)
        g = make()
        with GpuSolver(g, k) as s:
            s.set_policy(params)
            srcs = G.pick_sources(g, 3, 99).tolist() if k == 1 else [tuple(G.uniform_vertices(g.n, k, 2026).tolist())]
            rows = []
            for src in srcs:
                fixed = GpuOptions(**{**base.__dict__})
                learned = GpuOptions(**{**base.__dict__, "policy": Policy.Learned})
                tf = timed(s, src, fixed)
                tl = timed(s, src, learned)
                _, _, a = s.run_state(P._sources(src), fixed)
                sl, _, b = s.run_state(P._sources(src), learned)
                _, _, tr = P.run_traced(s, src, learned)
                rows.append({"src": src if k == 1 else f"batch of {k}", "fixed_ms": round(tf, 4), "learned_ms": round(tl, 4),
                             "speedup": round(tf / tl, 3), "bit_exact": bool(np.array_equal(a, b)),
                             "learned_buckets": sl.buckets,
                             "learned_deltas": [int(x) for x in tr[:, P.IN + 1]],
                             "learned_rounds_per_bucket": [int(x) for x in tr[:, P.IN + 3]]})
            report["eval"][name] = rows
            sp = statistics.median(r["speedup"] for r in rows)
            print(f"[eval] {name}: median speedup {sp:.2f}x, bit-exact {all(r['bit_exact'] for r in rows)}", flush=True)
    if args.report:
        Path(args.report).write_text(json.dumps(report, indent=1))
    return report


if __name__ == "__main__":
    main(sys.argv[1:])
