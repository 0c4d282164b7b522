"""Edge cases on the GPU, bit-exact against the oracle: a single vertex, a graph
without arcs, distances that overflow 32 bits (unreachable, as in the
reference's u64 sum compared with its u32 INF), A* from a vertex to itself,
duplicate sources in one batch."""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import GpuAlgo, GpuOptions, Schedule

pytestmark = pytest.mark.gpu

OPTS = [GpuOptions(schedule=Schedule.Async), GpuOptions(schedule=Schedule.Rounds),
        GpuOptions(algo=GpuAlgo.Frontier), GpuOptions(algo=GpuAlgo.NaiveRelax)]


@pytest.mark.parametrize("opt", OPTS)
def test_single_vertex_and_no_arcs(opt):
    g1 = pf.buildCSR(1, [], [], [])
    with pf.GpuSolver(g1, 1) as s:
        r = s.sssp(0, opt)
        assert list(r.dist) == [0] and list(r.parent) == [pf.NO_PARENT]
    g5 = pf.buildCSR(5, [], [], [])
    with pf.GpuSolver(g5, 1) as s:
        r = s.sssp(3, opt)
        assert list(r.dist) == [pf.INF_DIST] * 3 + [0, pf.INF_DIST]


@pytest.mark.parametrize("opt", OPTS)
def test_distances_beyond_32_bits_are_unreachable(oracle, opt):
    big = 0xFFFFFFFE
    g = pf.buildCSR(4, [0, 1, 0, 2], [1, 2, 3, 3], [2**31, 2**31, big, 1])
    with pf.GpuSolver(g, 1) as s:
        r = s.sssp(0, opt)
    d_ref, p_can = oracle.sssp_canonical(g, 0)
    assert np.array_equal(r.dist, d_ref) and np.array_equal(r.parent, p_can)
    assert r.dist[2] == pf.INF_DIST and r.dist[3] == big


def test_astar_to_itself_and_duplicate_sources(oracle):
    g = pf.grid(30, 30, 4)
    with pf.GpuSolver(g, 3) as s:
        a = s.astar(17, 17, GpuOptions())
        assert a.targetDist == 0 and list(a.path) == [17]
        _, _, state = s.run_state([5, 5, 100], GpuOptions())
    d, p = pf.unpack(state)
    for i, src in enumerate((5, 5, 100)):
        d_ref, p_can = oracle.sssp_canonical(g, src)
        assert np.array_equal(d[i * g.n:(i + 1) * g.n], d_ref)
        assert np.array_equal(p[i * g.n:(i + 1) * g.n], p_can)


def test_copy_ranges_that_would_wrap_are_rejected():
    # first + count past 2^64 must not pass the range check (the kernel would read
    # before the state array); both copy entry points refuse without touching the device
    import ctypes as C
    from pathfinding_gpu_b200 import _native as N
    g = pf.grid(10, 10, 1)
    with pf.GpuSolver(g, 2) as s:
        s.sssp(0, GpuOptions())
        lib = s._lib
        out32 = np.zeros(4, np.uint32)
        out64 = np.zeros(4, np.uint64)
        huge = (1 << 64) - 1
        assert lib.pfg_copy_dist(s.handle, huge, 2, N.ptr(out32, N.u32)) == 1
        assert lib.pfg_copy_state(s.handle, huge, 2, N.ptr(out64, N.u64)) == 1
        assert lib.pfg_copy_dist(s.handle, 2 * g.n - 1, 2, N.ptr(out32, N.u32)) == 1
        assert lib.pfg_copy_dist(s.handle, 2 * g.n - 2, 2, N.ptr(out32, N.u32)) == 0
        assert lib.pfg_copy_state(s.handle, huge, 2, N.ptr(out64, N.u64)) == 1
        assert b"range outside the state" in lib.pfg_last_error()
