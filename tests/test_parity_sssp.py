"""GPU parity of SSSP / A* / multi-source against the oracle (bit-exact).

dist must equal the reference's cpuDijkstra; parent must equal the canonical
smallest-index tight predecessor (the value the packed (dist<<32|parent)
atomicMin converges to); every run must also pass the reference's three
verifySSSP checks. A* must return cpuDijkstra's target distance and a valid
path of that cost (A* parents are schedule dependent, so they are not compared).
"""
import itertools

import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import GpuAlgo, GpuOptions, Mapping, AtomicMode, Compaction, Schedule
from pathfinding_gpu_b200 import _native as N

pytestmark = pytest.mark.gpu

SEED = 2026


@pytest.fixture(scope="module")
def grid100():
    return pf.grid(100, 100, SEED)


@pytest.fixture(scope="module")
def grid100_solver(grid100):
    s = pf.GpuSolver(grid100, 17)
    yield s
    s.close()


@pytest.fixture(scope="module")
def rmat12():
    return pf.rmat(12, 16, seed=SEED)


@pytest.fixture(scope="module")
def rmat12_solver(rmat12):
    s = pf.GpuSolver(rmat12, 8)
    yield s
    s.close()


def sources_c0(g):
    # source 0 plus 16 uniform sources from the seed
    return [0] + pf.uniform_vertices(g.n, 16, SEED).tolist()


def check_sssp(oracle, g, src, res):
    d_ref, p_can = oracle.sssp_canonical(g, src)
    assert np.array_equal(res.dist, d_ref), f"dist mismatch from {src}: {np.flatnonzero(res.dist != d_ref)[:5]}"
    assert np.array_equal(res.parent, p_can), f"parent mismatch from {src}: {np.flatnonzero(res.parent != p_can)[:5]}"
    rep = oracle.verify_sssp(g, src, d_ref, res.dist, res.parent, 64, src)
    assert rep["errors"] == 0, rep


ALGOS = [GpuAlgo.DeltaStep, GpuAlgo.Frontier, GpuAlgo.NaiveRelax]


@pytest.mark.parametrize("algo", ALGOS)
def test_grid100_all_sources(oracle, grid100, grid100_solver, algo):
    for src in sources_c0(grid100):
        res = grid100_solver.sssp(src, GpuOptions(algo=algo))
        check_sssp(oracle, grid100, src, res)


SCHEDULES = [Schedule.Rounds, Schedule.Async, Schedule.Warp, Schedule.Instance]


@pytest.mark.parametrize("mapping,atomic", list(itertools.product(list(Mapping), list(AtomicMode))))
@pytest.mark.parametrize("schedule", SCHEDULES)
def test_grid100_variants(oracle, grid100, grid100_solver, mapping, atomic, schedule):
    for algo in (GpuAlgo.DeltaStep, GpuAlgo.Frontier):
        res = grid100_solver.sssp(77, GpuOptions(algo=algo, mapping=mapping, atomic=atomic, schedule=schedule))
        check_sssp(oracle, grid100, 77, res)


@pytest.mark.parametrize("delta", [1, 7, 60, 100, 120, 149, 150, 1000, 100000])
@pytest.mark.parametrize("schedule", SCHEDULES)
def test_grid100_delta_sweep(oracle, grid100, grid100_solver, delta, schedule):
    res = grid100_solver.sssp(4321, GpuOptions(delta=delta, schedule=schedule))
    check_sssp(oracle, grid100, 4321, res)
    assert res.stats.delta == delta


def test_async_buckets_take_one_barrier_per_bucket(grid100_solver):
    # a bucket is one drain: far fewer barrier epochs than relaxation rounds
    a = grid100_solver.sssp(0, GpuOptions(schedule=Schedule.Async)).stats
    r = grid100_solver.sssp(0, GpuOptions(schedule=Schedule.Rounds)).stats
    assert a.rounds <= a.buckets + 2 < r.rounds


@pytest.mark.parametrize("block", [32, 256, 1024])
def test_grid300_async_batch(oracle, block):
    # wider wavefronts: claimed lists / work queues overflow and spill into the ring
    g = pf.grid(300, 300, SEED)
    srcs = pf.uniform_vertices(g.n, 8, SEED + 3).tolist()
    refs = [oracle.sssp_canonical(g, src) for src in srcs]
    with pf.GpuSolver(g, 8) as s:
        for atomic in (AtomicMode.MinRBA, AtomicMode.MinNoCheck):
            for sched in (Schedule.Async, Schedule.Warp, Schedule.Instance):
                _, _, state = s.run_state(srcs, GpuOptions(blockSize=block, atomic=atomic, schedule=sched))
                dist, parent = pf.unpack(state)
                for i, (d_ref, p_can) in enumerate(refs):
                    assert np.array_equal(dist[i * g.n:(i + 1) * g.n], d_ref), (block, atomic, sched, i)
                    assert np.array_equal(parent[i * g.n:(i + 1) * g.n], p_can), (block, atomic, sched, i)


def _check_batch(oracle, g, srcs, state):
    dist, parent = pf.unpack(state)
    for i, src in enumerate(srcs):
        d_ref, p_can = oracle.sssp_canonical(g, src)
        assert np.array_equal(dist[i * g.n:(i + 1) * g.n], d_ref), i
        assert np.array_equal(parent[i * g.n:(i + 1) * g.n], p_can), i


@pytest.mark.parametrize("k", [2, 3, 17, 64, 130])
def test_instance_windows_grid(oracle, k):
    # a bucket window per instance: every instance's own far piles, window advances and
    # hand-over of pending units (k >= 64: CTAs hold entries of many instances at once;
    # k = 130: the automatic schedule's own choice); duplicate sources and a Delta equal
    # to the largest weight (the smallest that applies)
    g = pf.grid(120, 90, SEED + 11)
    srcs = pf.uniform_vertices(g.n, k, SEED + k).tolist()
    srcs[-1] = srcs[0]
    maxw = int(g.maxW)
    with pf.GpuSolver(g, k) as s:
        for delta in (0, maxw, 4 * maxw):
            for block in (64, 256):
                stats, _, state = s.run_state(srcs, GpuOptions(delta=delta, blockSize=block,
                                                               schedule=Schedule.Instance))
                _check_batch(oracle, g, srcs, state)
                assert stats.buckets >= k  # every instance's first window counts
        # the automatic schedule (independent windows from 96 sources) and a shared window;
        # a window per instance counts at least one window per instance, a shared window
        # far fewer buckets than that on this graph
        for sched in (Schedule.Auto, Schedule.Async):
            stats, _, state = s.run_state(srcs, GpuOptions(schedule=sched))
            _check_batch(oracle, g, srcs, state)
            per_instance = sched == Schedule.Auto and k >= 96
            assert (stats.buckets >= k) == per_instance or k <= 17, (sched, k, stats.buckets)


def test_instance_windows_at_the_instance_limit(oracle):
    # 256 instances (the most one run takes with a window each; every CTA holds many of
    # them at once) and 257 (a shared window): identical results, checked on a sample
    g = pf.grid(60, 50, SEED + 21)
    srcs = pf.uniform_vertices(g.n, 257, SEED + 22).tolist()
    check = [0, 1, 127, 200, 255]
    with pf.GpuSolver(g, 257) as s:
        for k in (256, 257):
            stats, _, state = s.run_state(srcs[:k], GpuOptions(schedule=Schedule.Instance))
            dist, parent = pf.unpack(state)
            for i in check:
                d_ref, p_can = oracle.sssp_canonical(g, srcs[i])
                assert np.array_equal(dist[i * g.n:(i + 1) * g.n], d_ref), (k, i)
                assert np.array_equal(parent[i * g.n:(i + 1) * g.n], p_can), (k, i)
            # a window per instance counts every instance's windows; a shared one its buckets
            assert (stats.buckets >= k) == (k <= 256), (k, stats.buckets)


def test_instance_windows_fallbacks_and_long_rows(oracle, rmat12, rmat12_solver):
    # R-MAT rows above 32 arcs go through the CTA-cooperative dealing (the window word
    # travels in shared memory); Delta below the largest weight and the learned-policy
    # exclusions fall back to one shared window; results are identical either way
    srcs = [int(v) for v in pf.pick_sources(rmat12, 8, SEED + 5)]
    maxw = int(rmat12.maxW)
    for delta in (maxw, 3 * maxw, 16):
        for atomic in (AtomicMode.MinRBA, AtomicMode.CasRBA, AtomicMode.MinNoCheck):
            _, _, state = rmat12_solver.run_state(srcs, GpuOptions(delta=delta, atomic=atomic,
                                                                   schedule=Schedule.Instance))
            _check_batch(oracle, rmat12, srcs, state)


def test_instance_windows_repeated_runs(oracle, grid100, grid100_solver):
    # far stamps continue across runs of every schedule: alternate them on one solver
    srcs = sources_c0(grid100)
    for rep in range(3):
        for sched in (Schedule.Instance, Schedule.Async, Schedule.Rounds, Schedule.Instance):
            _, _, state = grid100_solver.run_state(srcs, GpuOptions(schedule=sched))
            _check_batch(oracle, grid100, srcs, state)
        check_sssp(oracle, grid100, 77, grid100_solver.sssp(77, GpuOptions(schedule=Schedule.Instance)))


@pytest.mark.parametrize("eager", [0, 1, 3, 16, 64])
def test_grid100_eager_subrounds(oracle, grid100, grid100_solver, eager):
    # in-round propagation changes the schedule only: results stay bit-exact
    for algo in (GpuAlgo.DeltaStep, GpuAlgo.Frontier):
        for src in (0, 5050, 9999):
            res = grid100_solver.sssp(src, GpuOptions(algo=algo, eager=eager))
            check_sssp(oracle, grid100, src, res)


def test_rmat_eager_subrounds(oracle, rmat12, rmat12_solver):
    s = int(pf.pick_sources(rmat12, 1, 11)[0])
    for eager in (0, 2, 32):
        for delta in (0, 8):
            check_sssp(oracle, rmat12, s, rmat12_solver.sssp(s, GpuOptions(eager=eager, delta=delta)))


def test_grid100_prefix_scan(oracle, grid100, grid100_solver):
    res = grid100_solver.sssp(5, GpuOptions(algo=GpuAlgo.Frontier, compaction=Compaction.PrefixScan))
    check_sssp(oracle, grid100, 5, res)


@pytest.mark.parametrize("block", [32, 64, 128, 256, 512, 1024, 100])
def test_grid100_block_sizes(oracle, grid100, grid100_solver, block):
    res = grid100_solver.sssp(9999, GpuOptions(blockSize=block))
    check_sssp(oracle, grid100, 9999, res)


def test_grid100_astar(oracle, grid100, grid100_solver):
    rng = pf.SplitMix64(SEED + 5)
    for _ in range(24):
        s, t = rng.below(grid100.n), rng.below(grid100.n)
        d_ref, _, _, _ = oracle.dijkstra(grid100, s)
        d_a, path_a, _, _ = oracle.astar(grid100, s, t)
        assert d_a == d_ref[t]
        for algo in ALGOS:
            r = grid100_solver.astar(s, t, GpuOptions(algo=algo))
            assert r.targetDist == d_ref[t], (s, t, algo)
            assert oracle.validate_path(grid100, r.path, s, t, int(d_ref[t])), (s, t, algo)
        for schedule, delta in itertools.product(SCHEDULES, (0, 60)):
            r = grid100_solver.astar(s, t, GpuOptions(schedule=schedule, delta=delta))
            assert r.targetDist == d_ref[t], (s, t, schedule, delta)
            assert oracle.validate_path(grid100, r.path, s, t, int(d_ref[t])), (s, t, schedule, delta)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_grid100_multisource(oracle, grid100, grid100_solver, schedule):
    srcs = sources_c0(grid100)
    for algo in (GpuAlgo.DeltaStep, GpuAlgo.Frontier):
        stats, ms, state = grid100_solver.run_state(srcs, GpuOptions(algo=algo, schedule=schedule))
        dist, parent = pf.unpack(state)
        dist = dist.reshape(len(srcs), -1)
        parent = parent.reshape(len(srcs), -1)
        for i, s in enumerate(srcs):
            d_ref, p_can = oracle.sssp_canonical(grid100, s)
            assert np.array_equal(dist[i], d_ref), (algo, i)
            assert np.array_equal(parent[i], p_can), (algo, i)


def test_multisource_dist_out_split_on_device(oracle, grid100, grid100_solver):
    # multiSource with distOut copies only the distance halves (split on the
    # device); any sub-range, odd starts included, matches the packed words
    srcs = sources_c0(grid100)
    dist_out = []
    grid100_solver.multiSource(srcs, GpuOptions(), dist_out)
    assert len(dist_out) == len(srcs)
    for i, s in enumerate(srcs):
        assert np.array_equal(dist_out[i], oracle.sssp_canonical(grid100, s)[0]), i
    state = np.empty(len(srcs) * grid100.n, np.uint64)
    N.check(grid100_solver._lib.pfg_copy_state(grid100_solver.handle, 0, state.size, N.ptr(state, N.u64)))
    for first, count in ((0, state.size), (1, 3), (grid100.n - 1, 2 * grid100.n + 5), (state.size - 1, 1),
                         (7, 0)):
        got = grid100_solver.copy_dist(first, count)
        assert np.array_equal(got, (state[first:first + count] >> np.uint64(32)).astype(np.uint32))
    with pytest.raises(pf.PfgError):
        grid100_solver.copy_dist(state.size - 1, 2)


def test_streamed_multisource(oracle, grid100, grid100_solver):
    # runs whose distance copies overlap the next run's kernel: every run's
    # distances equal the oracle, and a plain run after the stream is unaffected
    batches = [sources_c0(grid100), [5, 77, 9999], pf.uniform_vertices(grid100.n, 17, 7).tolist(), [1234]]
    outs = [np.full(len(b) * grid100.n, 7, np.uint32) for b in batches]
    for b, o in zip(batches, outs):
        grid100_solver.run_dist_async(b, o, GpuOptions(atomic=AtomicMode.MinNoCheck))
    grid100_solver.dist_wait()
    grid100_solver.dist_wait()  # nothing left: a no-op
    for b, o in zip(batches, outs):
        for i, s in enumerate(b):
            assert np.array_equal(o[i * grid100.n:(i + 1) * grid100.n], oracle.sssp_canonical(grid100, s)[0]), (b, i)
    grid100_solver.run_dist_async([3, 4], outs[1], GpuOptions())
    check_sssp(oracle, grid100, 42, grid100_solver.sssp(42, GpuOptions()))  # completes the stream first
    for i, s in enumerate([3, 4]):
        assert np.array_equal(outs[1][i * grid100.n:(i + 1) * grid100.n], oracle.sssp_canonical(grid100, s)[0])
    with pytest.raises(pf.PfgError):
        grid100_solver.run_dist_async(list(range(18)), np.empty(18 * grid100.n, np.uint32))


def test_rmat_variants(oracle, rmat12, rmat12_solver):
    srcs = pf.pick_sources(rmat12, 4, SEED)
    for algo, mapping in itertools.product(ALGOS, list(Mapping)):
        for s in srcs[:2]:
            res = rmat12_solver.sssp(int(s), GpuOptions(algo=algo, mapping=mapping))
            check_sssp(oracle, rmat12, int(s), res)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_rmat_small_delta_heavy_phase(oracle, rmat12, rmat12_solver, schedule):
    # Delta below the max weight exercises the R set and heavy rounds
    src = int(pf.pick_sources(rmat12, 1, 7)[0])
    for delta in (1, 16, 64, 200):
        res = rmat12_solver.sssp(src, GpuOptions(delta=delta, schedule=schedule))
        check_sssp(oracle, rmat12, src, res)
        assert res.stats.buckets >= 1


def test_errors_like_reference(grid100_solver):
    with pytest.raises(RuntimeError):
        grid100_solver.sssp(10**6, GpuOptions())
    with pytest.raises(RuntimeError):
        grid100_solver.astar(0, 10**6, GpuOptions())
    with pytest.raises(RuntimeError):
        grid100_solver.multiSource(list(range(18)), GpuOptions(), None)
    # the solver stays usable after an error
    assert grid100_solver.sssp(0, GpuOptions()).dist[0] == 0


@pytest.fixture(scope="module")
def hub_graph():
    # random arcs plus three long rows (25,000 / 9,000 / 3,000 arcs), so rows
    # exceed 8 x the block size and take the grid tier of the hybrid mapping
    rng = np.random.default_rng(7)
    n = 30000
    src = [rng.integers(0, n, 200000)]
    dst = [rng.integers(0, n, 200000)]
    for h, L in ((0, 25000), (17, 9000), (12345, 3000)):
        src.append(np.full(L, h))
        dst.append(rng.integers(0, n, L))
    src = np.concatenate(src).astype(np.uint32)
    dst = np.concatenate(dst).astype(np.uint32)
    w = rng.integers(1, 200, len(src)).astype(np.uint32)
    x = rng.uniform(0, 1000, n)
    y = rng.uniform(0, 1000, n)
    return pf.buildCSR(n, src, dst, w, x, y)


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("block,atomic", [(32, AtomicMode.MinRBA), (64, AtomicMode.MinNoCheck),
                                          (256, AtomicMode.MinRBA), (256, AtomicMode.CasRBA),
                                          (1024, AtomicMode.MinNoCheck)])
def test_hub_rows_grid_tier(oracle, hub_graph, schedule, block, atomic):
    g = hub_graph
    with pf.GpuSolver(g, 4) as s:
        for src in (0, 17, 5):
            for delta in (0, 20):
                res = s.sssp(src, GpuOptions(blockSize=block, atomic=atomic, schedule=schedule, delta=delta))
                check_sssp(oracle, g, src, res)
        srcs = [0, 17, 12345, 9]
        _, _, state = s.run_state(srcs, GpuOptions(blockSize=block, atomic=atomic, schedule=schedule))
        dist, parent = pf.unpack(state)
        for i, src in enumerate(srcs):
            d_ref, p_can = oracle.sssp_canonical(g, src)
            assert np.array_equal(dist[i * g.n:(i + 1) * g.n], d_ref), (schedule, block, i)
            assert np.array_equal(parent[i * g.n:(i + 1) * g.n], p_can), (schedule, block, i)


def test_hub_rows_astar_and_batch(oracle, hub_graph):
    from pathfinding_gpu_b200.batch import GpuBatch
    g = hub_graph
    with pf.GpuSolver(g, 1) as s:
        for src, dst in ((0, 29999), (17, 4), (12345, 100)):
            d_ref = oracle.dijkstra(g, src)[0]
            for schedule in SCHEDULES:
                r = s.astar(src, dst, GpuOptions(blockSize=64, schedule=schedule))
                assert r.targetDist == d_ref[dst]
                if d_ref[dst] != 0xFFFFFFFF:
                    assert oracle.validate_path(g, r.path, src, dst, int(d_ref[dst]))
    small = pf.grid(20, 20, 3)
    with GpuBatch([g, small], max_instances=4, max_states=3 * g.n + small.n) as b:
        inst = [(0, 0), (1, 5), (0, 17), (0, 12345)]
        b.set_instances(inst)
        for schedule in SCHEDULES:
            b.run(GpuOptions(blockSize=128, schedule=schedule))
            state = b.state()
            for i, (gi, src) in enumerate(inst):
                d, p = b.instance_result(i, state)
                d_ref, p_can = oracle.sssp_canonical([g, small][gi], src)
                assert np.array_equal(d, d_ref) and np.array_equal(p, p_can), (schedule, i)
