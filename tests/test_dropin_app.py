"""The drop-in proof on the GPU: the reference's own application (src/main.cpp and its
graph / CPU / verify / report sources, unchanged) linked against this repository's
include/gpu_sssp.h and GpuSolver (pathfinding_gpu_b200/csrc/gpu_solver.cpp) over
libpfg_b200.so, built by `make -C oracle pathfinder` into oracle/_ref/pathfinder_b200.

Its --mode verify runs every GPU SSSP variant (algorithms x mappings x atomic modes,
multi-source with distOut) and A* (reconstructPath on the returned parents) per source
and checks each against its own cpuDijkstra / cpuAStar with verifySSSP / validatePath;
it exits with 3 on any error (src/main.cpp:272-358, 875-994). The application is run on
its own grid and R-MAT generators, and in its single-query and multi-source modes.
"""
import os
import re
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
APP = ROOT / "oracle" / "_ref" / "pathfinder_b200"

if not APP.exists():
    pytestmark = [pytest.mark.gpu, pytest.mark.skip(reason="oracle/_ref/pathfinder_b200 not built "
                                                           "(make -C oracle pathfinder needs the reference's sources)")]


def run_app(tmp_path, *args, timeout=600):
    cmd = [str(APP), *args, "--out", str(tmp_path), "--no-color"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=dict(os.environ))
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("graph,n", [("grid", 40000), ("rmat", 1 << 15)])
def test_reference_verify_mode_passes(tmp_path, graph, n):
    rc, out = run_app(tmp_path, "--mode", "verify", "--graph", graph, "--n", str(n), "--queries", "3")
    assert rc == 0, out[-4000:]
    # the harness printed its checks and found no error
    assert re.search(r"(?i)pass", out), out[-2000:]
    assert not re.search(r"(?i)\bFAIL", out), out[-4000:]


def test_reference_single_astar_and_multisource(tmp_path):
    rc, out = run_app(tmp_path, "--mode", "single", "--graph", "grid", "--n", "250000", "--astar",
                      "--src", "17", "--dst", "240000", "--print-path")
    assert rc == 0, out[-4000:]
    rc, out = run_app(tmp_path, "--mode", "multisource", "--graph", "grid", "--n", "40000", "--batch", "8")
    assert rc == 0, out[-4000:]
