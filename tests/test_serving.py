"""Continuous-batching A* server: every answer equals the oracle's shortest distance,
and each query's answer is the same served alone and served in a mix of queries
admitted at different times (integers: no tolerance)."""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200.serving import GpuServer, run_poisson

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def road():
    return pf.road(64, seed=2026)


def pairs_for(g, k, seed):
    v = pf.uniform_vertices(g.n, 2 * k, seed)
    return [(int(v[2 * i]), int(v[2 * i + 1])) for i in range(k)]


def oracle_dist(oracle, g, pairs):
    return [int(oracle.dijkstra(g, s)[0][t]) for s, t in pairs]


def test_alone_equals_mix_equals_oracle(oracle, road):
    pairs = pairs_for(road, 24, 5)
    want = oracle_dist(oracle, road, pairs)
    with GpuServer(road, slots=8) as srv:
        alone = []
        for s, t in pairs:
            srv.submit(s, t)
            res = srv.drain(max_rounds=16)
            assert len(res) == 1
            alone.append(res[0]["dist"])
        assert alone == want
        # the same queries in a mix: admitted in waves while others are in flight
        ids = {}
        got = {}
        for wave in range(3):
            for s, t in pairs[wave * 8:(wave + 1) * 8]:
                ids[srv.submit(s, t)] = (s, t)
            srv.step(max_rounds=6)
            for r in srv.results():
                got[r["id"]] = r["dist"]
        for r in srv.drain(max_rounds=16):
            got[r["id"]] = r["dist"]
        mix = [got[q] for q in sorted(ids)]
        assert mix == want


def test_more_queries_than_slots_and_unreachable(oracle):
    a, b = pf.grid(12, 12, 1), pf.grid(6, 6, 2)
    g, offs = pf.union([a, b])
    pairs = [(0, 143), (5, 144 + 7), (144, 144 + 35), (3, 3), (150, 10)] * 3
    want = oracle_dist(oracle, g, pairs)
    with GpuServer(g, slots=3) as srv:
        for s, t in pairs:
            srv.submit(s, t)
        res = sorted(srv.drain(max_rounds=8), key=lambda r: r["id"])
    assert [r["dist"] for r in res] == want
    assert want[1] == 0xFFFFFFFF and want[3] == 0


def test_poisson_stream_latencies(oracle, road):
    pairs = pairs_for(road, 64, 9)
    want = dict(zip(range(len(pairs)), oracle_dist(oracle, road, pairs)))
    with GpuServer(road, slots=16) as srv:
        rep = run_poisson(srv, pairs, rate_qps=2000.0, max_rounds=8, seed=1)
    assert rep["queries"] == len(pairs)
    got = {r["id"] - 1: r["dist"] for r in rep["results"]}
    assert got == want
    assert 0 < rep["p50_ms"] <= rep["p99_ms"]


def test_answer_all_in_query_order(oracle, road):
    # the per-replica answer function of serve_sharded: distances in query order
    from pathfinding_gpu_b200.serving import answer_all
    v = pf.uniform_vertices(road.n, 2 * 12, 77)
    pairs = [(int(v[2 * i]), int(v[2 * i + 1])) for i in range(12)]
    with GpuServer(road, slots=5) as srv:
        got = answer_all(srv, pairs)
    assert got == [int(oracle.dijkstra(road, s)[0][t]) for s, t in pairs]


def test_slots_by_device_memory(oracle, road):
    # slots = 0: the server sizes itself by free device memory; answers stay exact
    pairs = pairs_for(road, 40, 21)
    want = oracle_dist(oracle, road, pairs)
    with GpuServer(road, slots=0) as srv:
        assert 1 <= srv.slots <= 2048 and srv.slots * road.n < 2 ** 32
        ids = [srv.submit(s, t) for s, t in pairs]
        got = {r["id"]: r["dist"] for r in srv.drain(max_rounds=8)}
    assert [got[q] for q in ids] == want


@pytest.mark.parametrize("schedule", ["Async", "Warp", "Rounds"])
def test_learned_policy_and_schedules_serve_the_same_answers(oracle, road, schedule):
    # the learned policy (when a network is loaded) and every drain change the
    # schedule only; without a network the server falls back to the fixed Delta
    from pathfinding_gpu_b200 import GpuOptions, Policy, Schedule
    from pathfinding_gpu_b200 import policy as P
    pairs = pairs_for(road, 24, 33)
    want = oracle_dist(oracle, road, pairs)
    opt = GpuOptions(policy=Policy.Learned, schedule=Schedule[schedule])
    with GpuServer(road, slots=6, opt=opt) as srv:
        ids = [srv.submit(s, t) for s, t in pairs[:12]]
        got = {r["id"]: r["dist"] for r in srv.drain(max_rounds=8)}  # no network yet: fixed Delta
        if P.WEIGHTS.exists():
            srv.set_policy(P.load())
        ids += [srv.submit(s, t) for s, t in pairs[12:]]
        got.update({r["id"]: r["dist"] for r in srv.drain(max_rounds=8)})
    assert [got[q] for q in ids] == want
