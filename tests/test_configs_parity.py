"""GPU parity at the benchmark configurations' own sizes, word for word against the oracle.

  * 1000 x 1000 grid (n = 10^6, m = 3,996,000): Naive, Frontier and Delta-stepping SSSP
    from source 0 and two seeded sources: dist equal to cpuDijkstra, parent equal to the
    canonical smallest-index tight predecessor, and the reference's verifySSSP checks;
  * the same grid's 256 point-to-point A* queries (pairs uniform from the seed): target
    distance equal to cpuAStar's (itself checked against cpuDijkstra on a sample) and every
    returned path valid for that distance (validatePath);
  * R-MAT scale 20, edge factor 16: three sources word for word, single-source runs and one
    three-instance multi-source launch;
  * the 2048 x 2048 road-like serving graph: a sample of served A* queries against the
    oracle's cpuAStar (not against another run of this engine).

These follow the reference's runVerify (src/main.cpp:272-358: every SSSP variant and A*
per source checked against cpuDijkstra) at full size.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import AtomicMode, GpuAlgo, GpuOptions, Schedule

pytestmark = pytest.mark.gpu

SEED = 2026


@pytest.fixture(scope="module")
def grid1000():
    return pf.grid(1000, 1000, SEED)


@pytest.fixture(scope="module")
def grid1000_canonical(grid1000, oracle):
    srcs = [0] + pf.uniform_vertices(grid1000.n, 2, SEED).tolist()
    return {s: oracle.sssp_canonical(grid1000, s) for s in srcs}


def _check(oracle, g, src, dist, parent, ref, what):
    d_ref, p_can = ref
    assert np.array_equal(dist, d_ref), (what, src, np.flatnonzero(dist != d_ref)[:5])
    assert np.array_equal(parent, p_can), (what, src, np.flatnonzero(parent != p_can)[:5])
    rep = oracle.verify_sssp(g, src, d_ref, dist, parent, 64, src)
    assert rep["errors"] == 0, (what, rep)


@pytest.mark.parametrize("algo", [GpuAlgo.NaiveRelax, GpuAlgo.Frontier, GpuAlgo.DeltaStep])
def test_grid1000_single_source_modes(oracle, grid1000, grid1000_canonical, algo):
    with pf.GpuSolver(grid1000, 1) as s:
        for src, ref in grid1000_canonical.items():
            r = s.sssp(src, GpuOptions(algo=algo))
            _check(oracle, grid1000, src, r.dist, r.parent, ref, algo.name)
            if algo == GpuAlgo.DeltaStep:
                r = s.sssp(src, GpuOptions(algo=algo, schedule=Schedule.Rounds, atomic=AtomicMode.MinNoCheck))
                _check(oracle, grid1000, src, r.dist, r.parent, ref, "DeltaStep rounds")


def test_grid1000_256_astar_pairs(oracle, grid1000):
    pairs = pf.uniform_vertices(grid1000.n, 2 * 256, SEED + 7).reshape(-1, 2).tolist()
    # the oracle's cpuAStar answers, in parallel (the C calls release the GIL)
    with ThreadPoolExecutor(max_workers=8) as ex:
        ref = list(ex.map(lambda st: oracle.astar(grid1000, st[0], st[1])[0], pairs))
    # cpuAStar itself agrees with cpuDijkstra (sample)
    for (a, b), d in list(zip(pairs, ref))[:4]:
        assert oracle.dijkstra(grid1000, a)[0][b] == d
    got = []
    with pf.GpuSolver(grid1000, 1) as s:
        for (a, b), d in zip(pairs, ref):
            r = s.astar(a, b, GpuOptions())
            got.append(r.targetDist)
            assert r.targetDist == d, (a, b, r.targetDist, d)
            assert oracle.validate_path(grid1000, r.path, a, b, d), (a, b)
        # the rounds schedule and the naive sweep on a sample of the same pairs
        for (a, b), d in list(zip(pairs, ref))[:8]:
            for o in (GpuOptions(schedule=Schedule.Rounds), GpuOptions(algo=GpuAlgo.Frontier)):
                r = s.astar(a, b, o)
                assert r.targetDist == d and oracle.validate_path(grid1000, r.path, a, b, d), (a, b, o)
    assert len(got) == 256


def test_rmat20_three_sources_word_for_word(oracle):
    g = pf.rmat(20, 16, seed=SEED)
    srcs = pf.pick_sources(g, 3, SEED).tolist()
    refs = {s: oracle.sssp_canonical(g, s) for s in srcs}
    with pf.GpuSolver(g, 3) as s:
        for src in srcs:
            for o in (GpuOptions(), GpuOptions(blockSize=1024, atomic=AtomicMode.MinNoCheck),
                      GpuOptions(schedule=Schedule.Warp)):
                r = s.sssp(src, o)
                _check(oracle, g, src, r.dist, r.parent, refs[src], ("rmat20", o.blockSize))
        _, _, state = s.run_state(srcs, GpuOptions())
        dist, parent = pf.unpack(state)
        for i, src in enumerate(srcs):
            _check(oracle, g, src, dist[i * g.n:(i + 1) * g.n], parent[i * g.n:(i + 1) * g.n], refs[src],
                   "rmat20 multi-source")


def test_road2048_served_queries_against_the_oracle(oracle):
    from pathfinding_gpu_b200.serving import GpuServer
    road = pf.road(2048, seed=SEED)
    v = pf.uniform_vertices(road.n, 2 * 64, SEED + 11)
    pairs = [(int(v[2 * i]), int(v[2 * i + 1])) for i in range(64)]
    with GpuServer(road, slots=32) as srv:
        ids = {srv.submit(a, t): (a, t) for a, t in pairs}
        got = {r["id"]: r for r in srv.drain(max_rounds=8)}
    assert len(got) == len(pairs)
    sample = list(ids.items())[:24]
    with ThreadPoolExecutor(max_workers=8) as ex:
        ref = list(ex.map(lambda it: oracle.astar(road, it[1][0], it[1][1])[0], sample))
    for (q, (a, t)), d in zip(sample, ref):
        assert got[q]["dist"] == d, (a, t, got[q]["dist"], d)
