"""Failure handling without a GPU fault: every device-side wait is bounded.

With PFG_TEST_ABSENT_CTA=1 the persistent kernel's CTA 0 leaves at once, so no
grid barrier can complete; every other CTA's wait runs into the PFG_TIMEOUT_MS
limit, the run ends with PFG_ERR_DEVICE_TIMEOUT (status 5), and the context
and the solver stay usable: the next run is bit-exact again."""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import GpuAlgo, GpuOptions, Schedule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("opt", [GpuOptions(schedule=Schedule.Rounds), GpuOptions(schedule=Schedule.Async),
                                 GpuOptions(algo=GpuAlgo.Frontier)])
def test_barrier_wait_times_out_and_solver_recovers(oracle, monkeypatch, opt):
    g = pf.grid(40, 40, 3)
    with pf.GpuSolver(g, 2) as s:
        monkeypatch.setenv("PFG_TIMEOUT_MS", "100")
        monkeypatch.setenv("PFG_TEST_ABSENT_CTA", "1")
        with pytest.raises(RuntimeError) as e:
            s.sssp(5, opt)
        assert getattr(e.value, "status", None) == 5, e.value
        monkeypatch.delenv("PFG_TEST_ABSENT_CTA")
        r = s.sssp(5, opt)
        d_ref, p_can = oracle.sssp_canonical(g, 5)
        assert np.array_equal(r.dist, d_ref) and np.array_equal(r.parent, p_can)
        stats, ms, state = s.run_state([7, 1500], opt)
        d, p = pf.unpack(state)
        for i, src in enumerate((7, 1500)):
            d_ref, p_can = oracle.sssp_canonical(g, src)
            assert np.array_equal(d[i * g.n:(i + 1) * g.n], d_ref)
            assert np.array_equal(p[i * g.n:(i + 1) * g.n], p_can)


def test_instance_windows_run_times_out_and_solver_recovers(oracle, monkeypatch):
    # a multi-source run under independent windows that fails: the solver clears its stamp
    # words before the next run (the failed drain may have used far epochs it never recorded)
    g = pf.grid(40, 40, 3)
    srcs = [7, 1500, 800]
    opt = GpuOptions(schedule=Schedule.Instance)
    with pf.GpuSolver(g, 3) as s:
        for _ in range(2):
            _, _, state = s.run_state(srcs, opt)
        monkeypatch.setenv("PFG_TIMEOUT_MS", "100")
        monkeypatch.setenv("PFG_TEST_ABSENT_CTA", "1")
        with pytest.raises(RuntimeError) as e:
            s.run_state(srcs, opt)
        assert getattr(e.value, "status", None) == 5, e.value
        monkeypatch.delenv("PFG_TEST_ABSENT_CTA")
        for sched in (Schedule.Instance, Schedule.Async, Schedule.Instance):
            _, _, state = s.run_state(srcs, GpuOptions(schedule=sched))
            d, p = pf.unpack(state)
            for i, src in enumerate(srcs):
                d_ref, p_can = oracle.sssp_canonical(g, src)
                assert np.array_equal(d[i * g.n:(i + 1) * g.n], d_ref), (sched, i)
                assert np.array_equal(p[i * g.n:(i + 1) * g.n], p_can), (sched, i)


def test_long_progressing_drain_is_not_a_timeout(oracle, monkeypatch):
    # A 100,000-vertex path with one huge bucket: one CTA walks the chain for
    # far longer than the 100 ms wait limit while every other CTA waits. The
    # limit counts from the last progress anywhere, so the run succeeds.
    n = 100000
    src = np.arange(n - 1, dtype=np.uint32)
    g = pf.buildCSR(n, src, src + 1, np.full(n - 1, 3, np.uint32))
    monkeypatch.setenv("PFG_TIMEOUT_MS", "100")
    with pf.GpuSolver(g, 1) as s:
        r = s.sssp(0, GpuOptions(schedule=Schedule.Async, delta=1 << 30))
    assert r.dist[-1] == 3 * (n - 1) and r.parent[-1] == n - 2
    d_ref, p_can = oracle.sssp_canonical(g, 0)
    assert np.array_equal(r.dist, d_ref) and np.array_equal(r.parent, p_can)
