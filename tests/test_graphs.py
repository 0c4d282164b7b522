"""Host graph substrate (pfg_graphs.cpp): generators of the benchmark workloads, the
weight-sorted CSR builder (checked against the oracle's restatement of the
reference's buildCSR), and the DIMACS / SNAP / PFCSR001 loaders. CPU only."""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf


def arcs_of(g):
    src = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(g.row_offsets))
    return src, g.col_indices, g.weights


def assert_csr_contract(g):
    row, col, w = g.row_offsets, g.col_indices, g.weights
    assert row[0] == 0 and row[-1] == g.m and np.all(np.diff(row.astype(np.int64)) >= 0)
    assert np.all(col < g.n) and np.all(w >= 1)
    src = np.repeat(np.arange(g.n), np.diff(row))
    assert not np.any(src == col), "self loop"
    key = (src.astype(np.uint64) << np.uint64(40)) | (w.astype(np.uint64) << np.uint64(20)) | col
    if g.n < (1 << 20) and w.max() < (1 << 20):
        assert np.all(np.diff(key.astype(np.int64)) >= 0), "rows not sorted by (w, dst)"


def test_grid_workload_c0():
    g = pf.grid(100, 100, 2026)
    assert (g.n, g.m) == (10000, 39600)
    assert g.hScale == 100.0 and g.minW >= 100 and g.maxW <= 150
    assert_csr_contract(g)
    assert g.x[101] == 1.0 and g.y[101] == 1.0


def test_grid_workload_c1_size():
    g = pf.grid(1000, 1000, 2026)
    assert (g.n, g.m) == (1_000_000, 3_996_000)


def test_rmat_workload_properties():
    g = pf.rmat(12, 16, seed=2026)
    assert g.n == 4096 and g.x is None
    assert_csr_contract(g)
    assert g.minW >= 1 and g.maxW <= 255
    src, dst, _ = arcs_of(g)
    pairs = src.astype(np.uint64) << np.uint64(32) | dst
    assert len(np.unique(pairs)) == g.m, "duplicate arcs must be merged"
    assert g.maxDeg > 10 * g.avgDeg  # power-law degrees


def test_rmat_duplicates_keep_the_lightest_copy():
    # regenerate the same samples through the generic builder and compare
    g = pf.rmat(8, 8, seed=5)
    src, dst, w = arcs_of(g)
    d = {}
    for s, t, x in zip(src.tolist(), dst.tolist(), w.tolist()):
        assert (s, t) not in d
        d[(s, t)] = x
    assert len(d) == g.m


def test_road_workload_c4_small():
    g = pf.road(128, seed=2026)
    assert g.n == 128 * 128
    assert_csr_contract(g)
    assert g.hScale == 100.0
    full = 4 * 128 * 127
    assert 0.85 * full < g.m < 0.95 * full + 0.03 * g.n


def test_grid_batch_sides():
    sides = pf.grid_batch_sides(256, 32, 316, 2026)
    assert len(sides) == 256 and min(sides) >= 32 and max(sides) <= 316
    assert len(set(sides)) > 50


def test_builder_matches_the_oracle_restatement(oracle):
    rng = np.random.default_rng(3)
    n = 300
    s = rng.integers(0, n, 5000).astype(np.uint32)
    d = rng.integers(0, n, 5000).astype(np.uint32)
    w = rng.integers(0, 50, 5000).astype(np.uint32)  # zeros are clamped to 1
    x, y = rng.uniform(0, 100, n), rng.uniform(0, 100, n)
    g = pf.buildCSR(n, s, d, w, x, y)
    row, col, wt, st = oracle.build_csr(n, s, d, w, x, y)
    assert np.array_equal(g.row_offsets, row) and np.array_equal(g.col_indices, col)
    assert np.array_equal(g.weights, wt)
    assert g.hScale == st["hScale"] and g.avgW == st["avgW"] and g.maxDeg == st["maxDeg"]


def test_union_offsets_components():
    a, b = pf.grid(5, 5, 1), pf.grid(3, 4, 2)
    u, offs = pf.union([a, b])
    assert u.n == a.n + b.n and u.m == a.m + b.m and offs.tolist() == [0, a.n]
    assert np.array_equal(u.row_offsets[: a.n + 1], a.row_offsets)
    assert np.array_equal(u.col_indices[a.m:], b.col_indices + a.n)


def test_binary_cache_round_trip(tmp_path):
    g = pf.grid(20, 30, 7)
    p = tmp_path / "g.bin"
    g.save_binary(str(p))
    h = pf.load_binary(str(p))
    assert np.array_equal(g.row_offsets, h.row_offsets) and np.array_equal(g.col_indices, h.col_indices)
    assert np.array_equal(g.weights, h.weights) and np.array_equal(g.x, h.x) and h.hScale == g.hScale
    with open(p, "r+b") as f:
        f.write(b"XXXXXXXX")
    with pytest.raises(RuntimeError):
        pf.load_binary(str(p))


def test_dimacs_loader(tmp_path):
    gr = tmp_path / "t.gr"
    co = tmp_path / "t.co"
    gr.write_text("c comment\np sp 4 5\na 1 2 7\na 2 3 1\na 3 4 2\na 4 1 9\na 1 3 10\n")
    co.write_text("p aux sp co 4\nv 1 0 0\nv 2 1000000 0\nv 3 1000000 1000000\nv 4 0 1000000\n")
    g = pf.load_dimacs(str(gr), str(co))
    assert (g.n, g.m) == (4, 5)
    assert g.row_offsets.tolist() == [0, 2, 3, 4, 5]
    assert g.col_indices[:2].tolist() == [1, 2] and g.weights[:2].tolist() == [7, 10]
    assert g.x is not None and g.hScale > 0
    with pytest.raises(RuntimeError):
        bad = tmp_path / "bad.gr"
        bad.write_text("a 1 2 3\n")
        pf.load_dimacs(str(bad))


def test_snap_loader(tmp_path):
    p = tmp_path / "e.txt"
    p.write_text("# FromNodeId ToNodeId\n0 1\n1 2\n2 0 5\n% other comment\n3 3\n")
    g = pf.load_snap(str(p), symmetrize=True, max_w=1000, seed=2026)
    assert g.n == 4 and g.m == 6  # self loop 3->3 dropped, each arc mirrored
    w01 = g.weights[np.flatnonzero(g.col_indices[g.row_offsets[0]:g.row_offsets[1]] == 1)[0]]
    w10 = g.weights[g.row_offsets[1] + np.flatnonzero(g.col_indices[g.row_offsets[1]:g.row_offsets[2]] == 0)[0]]
    assert w01 == w10 and 1 <= w01 <= 1000


def test_oracle_restates_the_benchmark_grid():
    # the oracle's generator of the benchmark grid (used by bench.py's reference arm,
    # which must not load this library) builds the same CSR as pfg_graph_gen_grid
    from oracle import oracle as O
    for rows, cols, seed in ((100, 100, 2026), (37, 53, 5), (1000, 1000, 2026)):
        a = O.config_grid(rows, cols, seed)
        g = pf.grid(rows, cols, seed)
        assert np.array_equal(a.row_offsets, g.row_offsets) and np.array_equal(a.col_indices, g.col_indices)
        assert np.array_equal(a.weights, g.weights) and np.array_equal(a.x, g.x) and np.array_equal(a.y, g.y)
        assert a.hScale == g.hScale and a.stats["avgW"] == g.avgW
    assert np.array_equal(O.uniform_vertices(10 ** 6, 64, 2026), pf.uniform_vertices(10 ** 6, 64, 2026))
