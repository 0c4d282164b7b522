"""The schedule autotuner (pathfinding_gpu_b200/autotune.py) on the GPU.

tune() runs coordinate descent over launch shape, atomic mode, eager sub-rounds and
Delta multiplier with the engine's own CUDA-event times. The options it returns must
give states identical to the default options' (a schedule never changes results), its
recorded time must not exceed the default's (the default is its first candidate), and
the result must come back from the JSON cache keyed by the workload's signature.
"""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import GpuOptions, autotune

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["grid", "rmat"])
def test_tune_keeps_results_and_never_loses_to_the_default(tmp_path, monkeypatch, which):
    monkeypatch.setenv("PFG_TUNE_CACHE", str(tmp_path / "tune.json"))
    g = pf.grid(300, 300, 2026) if which == "grid" else pf.rmat(14, 16, seed=2026)
    srcs = pf.uniform_vertices(g.n, 4, 77).tolist() if which == "grid" else pf.pick_sources(g, 4, 77).tolist()
    with pf.GpuSolver(g, len(srcs)) as s:
        base = GpuOptions()
        _, _, want = s.run_state(srcs, base)
        time_fn = lambda o: s.run_state(srcs, o, copy=False)[1]
        key = autotune.signature(g, len(srcs), base.algo)
        best, best_ms, log = autotune.tune(time_fn, base, s.autoDelta(), reps=2, key=key)
        assert log, "no candidate was timed"
        default_ms = log[0][1]
        assert best_ms <= default_ms
        assert len(log) >= 8  # every knob was tried
        _, _, got = s.run_state(srcs, best)
        assert np.array_equal(got, want), f"tuned options {best} change the result"
        # the cache returns the same choice without timing anything
        again, ms2, log2 = autotune.tune(time_fn, base, s.autoDelta(), key=key)
        assert again == best and log2 == []
