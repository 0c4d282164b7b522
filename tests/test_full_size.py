"""The benchmark workloads at full size, checked through properties that prove the
result exact without a CPU run per instance (weights are positive):

  * d[source] = 0;
  * no arc is violated: d[v] <= d[u] + w for every arc with d[u] finite;
  * every reached vertex other than the source has a tight parent arc,
    d[v] = d[parent] + w(parent, v)  (so d is the shortest distance);
  * no tight arc (u, v) has u < parent[v]  (the parent is the canonical one, the
    smallest tight predecessor the packed atomicMin converges to).

A few instances are also compared word for word with the oracle."""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import AtomicMode, GpuOptions, Schedule

pytestmark = pytest.mark.gpu

INF = np.uint64(0xFFFFFFFF)


def arcs(g):
    deg = np.diff(g.row_offsets).astype(np.int64)
    return (np.repeat(np.arange(g.n, dtype=np.uint32), deg), g.col_indices, g.weights.astype(np.uint64))


def check_properties(A, src, dist, parent, what=""):
    u, v, w = A
    d = dist.astype(np.uint64)
    assert dist[src] == 0 and parent[src] == pf.NO_PARENT, (what, src, int(dist[src]), int(parent[src]))
    du, dv = d[u], d[v]
    fin = du != INF
    cand = du + w
    assert not np.any(fin & (cand < dv)), ("violated arc", what)
    tight = fin & (cand == dv)
    par = parent.astype(np.int64)
    tight_par = tight & (u.astype(np.int64) == par[v])
    reached = dist != 0xFFFFFFFF
    reached[src] = False
    has_par = np.zeros(len(dist), bool)
    has_par[v[tight_par]] = True
    assert np.array_equal(has_par, reached), ("reached vertex without a tight parent arc", what)
    assert not np.any(tight & (u.astype(np.int64) < par[v])), ("parent is not the smallest tight predecessor", what)


def test_grid1000_64_sources(oracle):
    g = pf.grid(1000, 1000, 2026)
    srcs = pf.uniform_vertices(g.n, 64, 2026).tolist()
    A = arcs(g)
    with pf.GpuSolver(g, 64) as s:
        for opt in (GpuOptions(atomic=AtomicMode.MinNoCheck), GpuOptions(schedule=Schedule.Rounds),
                    GpuOptions(atomic=AtomicMode.MinNoCheck, schedule=Schedule.Warp, blockSize=1024)):
            _, _, state = s.run_state(srcs, opt)
            dist, parent = pf.unpack(state)
            for i, src in enumerate(srcs):
                check_properties(A, src, dist[i * g.n:(i + 1) * g.n], parent[i * g.n:(i + 1) * g.n], i)
            for i in (0, 63):
                d_ref, p_can = oracle.sssp_canonical(g, srcs[i])
                assert np.array_equal(dist[i * g.n:(i + 1) * g.n], d_ref)
                assert np.array_equal(parent[i * g.n:(i + 1) * g.n], p_can)


def test_rmat20(oracle):
    g = pf.rmat(20, 16, seed=2026)
    A = arcs(g)
    srcs = pf.pick_sources(g, 3, 2026).tolist()
    with pf.GpuSolver(g, 3) as s:
        for opt in (GpuOptions(blockSize=1024), GpuOptions(), GpuOptions(delta=16, schedule=Schedule.Rounds),
                    GpuOptions(schedule=Schedule.Warp), GpuOptions(schedule=Schedule.Warp, delta=16)):
            _, _, state = s.run_state(srcs, opt)
            dist, parent = pf.unpack(state)
            for i, src in enumerate(srcs):
                check_properties(A, src, dist[i * g.n:(i + 1) * g.n], parent[i * g.n:(i + 1) * g.n], i)
        d_ref, p_can = oracle.sssp_canonical(g, srcs[0])
        assert np.array_equal(dist[:g.n], d_ref) and np.array_equal(parent[:g.n], p_can)


@pytest.mark.parametrize("schedule", [Schedule.Async, Schedule.Rounds, Schedule.Warp])
def test_uneven_batch_full_size(schedule):
    from pathfinding_gpu_b200.batch import GpuBatch
    big = pf.grid(1024, 1024, 2026)
    small = pf.grid_batch(256, 32, 316, 2026)
    graphs = [big] + small
    inst = [(0, int(v)) for v in pf.uniform_vertices(big.n, 64, 2026)]
    inst += [(i + 1, int(pf.uniform_vertices(gs.n, 1, 100 + i)[0])) for i, gs in enumerate(small)]
    states = 64 * big.n + sum(gs.n for gs in small)
    arcs_of = {}
    with GpuBatch(graphs, max_states=states, max_instances=len(inst)) as b:
        b.set_instances(inst)
        b.capture(GpuOptions(atomic=AtomicMode.MinNoCheck, schedule=schedule))
        b.replay()
        state = b.state()
        for i, (gi, src) in enumerate(inst):
            if gi not in arcs_of:
                arcs_of[gi] = arcs(graphs[gi])
            d, p = b.instance_result(i, state)
            check_properties(arcs_of[gi], src, d, p, (i, gi))


def test_road2048_astar_and_serving():
    from pathfinding_gpu_b200.serving import GpuServer
    road = pf.road(2048, seed=2026)
    A = arcs(road)
    v = pf.uniform_vertices(road.n, 2 * 48, 2026)
    pairs = [(int(v[2 * i]), int(v[2 * i + 1])) for i in range(48)]
    srcs = sorted({s for s, _ in pairs})
    want = {}
    with pf.GpuSolver(road, len(srcs)) as s:
        _, _, state = s.run_state(srcs, GpuOptions())
        dist, parent = pf.unpack(state)
        for i, src in enumerate(srcs):
            di = dist[i * road.n:(i + 1) * road.n]
            check_properties(A, src, di, parent[i * road.n:(i + 1) * road.n], i)
            want.update({(a, t): int(di[t]) for a, t in pairs if a == src})
        for a, t in pairs[:4]:
            r = s.astar(a, t, GpuOptions())
            assert r.targetDist == want[(a, t)]
    with GpuServer(road, slots=32) as srv:
        ids = {srv.submit(a, t): (a, t) for a, t in pairs}
        got = {r["id"]: r["dist"] for r in srv.drain(max_rounds=8)}
    assert len(got) == len(pairs)
    for q, (a, t) in ids.items():
        assert got[q] == want[(a, t)], (a, t)
