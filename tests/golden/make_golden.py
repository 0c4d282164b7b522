"""Generates tests/golden/ref_fixtures.npz from the reference's own CPU code.

Runs in a checkout where the reference sources are present: oracle/Makefile
compiles src/graph.cpp, src/cpu_sssp.cpp, src/verify.cpp, src/term.cpp of the
reference into oracle/_ref/libpfref.so; this script calls the reference's
genGridRoad / genRMAT / buildCSR / cpuDijkstra / cpuAStar / pickSources /
heuristicValue through it and stores their outputs. The fixtures pin the C
oracle (oracle/pfg_oracle.c) in tests/test_oracle.py, where the reference
itself is not available.

    python tests/golden/make_golden.py [--reference /path/to/reference]
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

SEED = 2026


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PFG_REFERENCE", str(ROOT.parent / "reference")),
                    help="reference checkout (default: $PFG_REFERENCE, else ../reference beside the repository)")
    args = ap.parse_args()
    O.build(args.reference)
    if not O.ref_available():
        raise SystemExit("reference shim not built")
    out = {}

    # 1. reference road grid (jitter, deletions, diagonals, arterials)
    rg = O.ref_gen_grid_road(30, 30, SEED)
    row, col, w, x, y, st = rg.arrays()
    out.update(road_row=row, road_col=col, road_w=w, road_x=x, road_y=y,
               road_stats=np.array([st["m"], st["minW"], st["maxW"], st["maxDeg"], st["avgW"], st["avgDeg"],
                                    st["hScale"]]))
    srcs = rg.pick_sources(3, SEED + 7)
    out["road_srcs"] = srcs
    dists, pars = [], []
    for s in srcs:
        d, p, _, _ = rg.dijkstra(int(s))
        dists.append(d)
        pars.append(p)
    out["road_dist"] = np.stack(dists)
    out["road_parent"] = np.stack(pars)
    pairs, adist, apath_len, apaths = [], [], [], []
    rng = np.random.default_rng(SEED)
    for i in range(6):
        s, t = (int(v) for v in rng.integers(0, row.shape[0] - 1, 2))
        d, path, _, _ = rg.astar(s, t, True)
        pairs.append((s, t))
        adist.append(d)
        apath_len.append(len(path))
        apaths.extend(path)
    out["road_astar_pairs"] = np.array(pairs, np.uint32)
    out["road_astar_dist"] = np.array(adist, np.uint32)
    out["road_astar_len"] = np.array(apath_len, np.uint32)
    out["road_astar_paths"] = np.array(apaths, np.uint32)

    # 2. reference R-MAT (undirected, permuted, hash weights)
    rm = O.ref_gen_rmat(10, 8, 1000, SEED)
    row, col, w, _, _, st = rm.arrays()
    out.update(rmat_row=row, rmat_col=col, rmat_w=w,
               rmat_stats=np.array([st["m"], st["minW"], st["maxW"], st["maxDeg"], st["avgW"], st["avgDeg"],
                                    st["hScale"]]))
    srcs = rm.pick_sources(2, SEED + 3)
    out["rmat_srcs"] = srcs
    out["rmat_dist"] = np.stack([rm.dijkstra(int(s))[0] for s in srcs])
    out["rmat_parent"] = np.stack([rm.dijkstra(int(s))[1] for s in srcs])

    # 3. the reference's buildCSR on an arc list with self loops, duplicates and w = 0
    n = 50
    s = rng.integers(0, n, 600).astype(np.uint32)
    d = rng.integers(0, n, 600).astype(np.uint32)
    ww = rng.integers(0, 20, 600).astype(np.uint32)
    xs = rng.uniform(0, 10, n)
    ys = rng.uniform(0, 10, n)
    bg = O.ref_build_csr(n, s, d, ww, xs, ys)
    row, col, w, _, _, st = bg.arrays()
    out.update(build_in_src=s, build_in_dst=d, build_in_w=ww, build_in_x=xs, build_in_y=ys,
               build_row=row, build_col=col, build_w=w,
               build_stats=np.array([st["m"], st["minW"], st["maxW"], st["maxDeg"], st["avgW"], st["avgDeg"],
                                     st["hScale"]]))

    # 4. heuristicValue samples
    pts = rng.uniform(-1e5, 1e5, (64, 5))
    pts[:, 4] = np.abs(pts[:, 4]) / 1e5
    out["heur_in"] = pts
    out["heur_out"] = np.array([O.ref().ref_heuristic(*map(float, p)) for p in pts], np.uint32)

    path = Path(__file__).resolve().parent / "ref_fixtures.npz"
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
