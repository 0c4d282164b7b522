#!/bin/bash
# TEST INFRASTRUCTURE - comparison runs, not part of the product.
#
# Runs the reference's own benchmark harness (src/main.cpp, --mode bench and
# --mode multisource) twice on the same graph files: once with the reference's
# CUDA engine compiled for sm_100a (oracle/_ref/pathfinder_ref, `make -C oracle
# refgpu`) and once with this repository's engine behind the reference's
# GpuSolver interface (oracle/_ref/pathfinder_b200, `make -C oracle pathfinder`).
# The harness verifies every GPU result against its CPU Dijkstra and writes its
# CSV files under OUT/ref and OUT/b200.
#
#   bash oracle/compare_reference_gpu.sh [OUT]    (graph files go to a temporary directory)
set -euo pipefail
OUT=${1:-compare_out}
HERE=$(cd "$(dirname "$0")" && pwd)
GRAPHS=$(mktemp -d)
trap 'rm -rf "$GRAPHS"' EXIT
mkdir -p "$OUT/ref" "$OUT/b200"
python -c "
import pathfinding_gpu_b200 as pf
pf.grid(1000, 1000, 2026).save_binary('$GRAPHS/grid1000.bin')
pf.rmat(20, 16, seed=2026).save_binary('$GRAPHS/rmat20.bin')
"
for B in ref b200; do
  for G in grid1000 rmat20; do
    "$HERE/_ref/pathfinder_$B" --mode bench --graph bin --file "$GRAPHS/$G.bin" --out "$OUT/$B" --no-color \
        > "$OUT/$B/bench_$G.log" 2>&1
  done
  "$HERE/_ref/pathfinder_$B" --mode multisource --graph bin --file "$GRAPHS/grid1000.bin" --batch 64 \
      --out "$OUT/$B" --no-color > "$OUT/$B/multisource_grid1000.log" 2>&1
done
echo "done: $OUT"
