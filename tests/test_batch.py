"""Uneven batches: many graphs and sources in one persistent launch (pfg_batch_*),
per-instance results bit-exact against the oracle, CUDA-graph replay identical."""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import GpuAlgo, GpuOptions, Schedule
from pathfinding_gpu_b200.batch import GpuBatch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs():
    return [pf.grid(30, 30, 1), pf.grid(17, 41, 2), pf.rmat(10, 8, seed=3), pf.grid(2, 2, 4)]


def check_instances(oracle, b, graphs, state):
    for i, (gi, s) in enumerate(b.instances):
        d, p = b.instance_result(i, state)
        d_ref, p_can = oracle.sssp_canonical(graphs[gi], s)
        assert np.array_equal(d, d_ref), (i, gi, s)
        assert np.array_equal(p, p_can), (i, gi, s)


@pytest.mark.parametrize("algo,schedule", [(GpuAlgo.DeltaStep, Schedule.Rounds), (GpuAlgo.DeltaStep, Schedule.Async),
                                           (GpuAlgo.Frontier, Schedule.Auto)])
def test_uneven_batch_matches_single_runs(oracle, graphs, algo, schedule):
    inst = [(0, 0), (0, 899), (0, 450), (1, 5), (2, 17), (2, 900), (3, 3), (1, 696)]
    with GpuBatch(graphs, max_instances=16, max_states=8 * 2000) as b:
        b.set_instances(inst)
        for delta in (0, 5, 200):
            stats, ms = b.run(GpuOptions(algo=algo, delta=delta, schedule=schedule))
            check_instances(oracle, b, graphs, b.state())
            assert stats.rounds > 0 and ms > 0


def test_capture_replay_identical(oracle, graphs):
    inst = [(1, 3), (0, 77), (2, 5), (2, 6)]
    with GpuBatch(graphs, max_instances=8, max_states=4000) as b:
        b.set_instances(inst)
        s1, _ = b.run(GpuOptions())
        st1 = b.state()
        b.capture(GpuOptions())
        for _ in range(3):
            s2, ms = b.replay()
            assert np.array_equal(b.state(), st1)
            assert s2.rounds == s1.rounds or s2.edgesScanned > 0
        check_instances(oracle, b, graphs, st1)
        b.set_instances([(0, 1)])  # a new table invalidates the recorded run
        with pytest.raises(RuntimeError):
            b.replay()


def test_batch_errors(graphs):
    with GpuBatch(graphs, max_instances=4, max_states=2000) as b:
        with pytest.raises(RuntimeError):
            b.set_instances([(9, 0)])
        with pytest.raises(RuntimeError):
            b.set_instances([(0, 900)])
        with pytest.raises(RuntimeError):
            b.set_instances([(0, 0), (0, 1), (0, 2)])  # 2700 states > 2000
        with pytest.raises(RuntimeError):
            b.set_instances([(3, 0)] * 5)  # more than max_instances
        b.set_instances([(3, 0)])
        b.run()
