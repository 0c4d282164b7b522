"""The C oracle against the reference: golden fixtures made by the reference's own
code (tests/golden/make_golden.py) and the graph statistics the reference printed
in its published logs. CPU only."""
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "ref_fixtures.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def graph(row, col, w, x=None, y=None, hscale=0.0):
    return SimpleNamespace(row_offsets=row, col_indices=col, weights=w, x=x, y=y, hScale=hscale)


def test_genGridRoad_and_buildCSR_reproduce_the_reference(oracle, gold):
    n, s, d, w, x, y = oracle.gen_grid_road(30, 30, 2026)
    row, col, wt, st = oracle.build_csr(n, s, d, w, x, y)
    assert np.array_equal(row, gold["road_row"])
    assert np.array_equal(col, gold["road_col"])
    assert np.array_equal(wt, gold["road_w"])
    assert np.array_equal(x, gold["road_x"]) and np.array_equal(y, gold["road_y"])
    ref = gold["road_stats"]
    assert [st["m"], st["minW"], st["maxW"], st["maxDeg"]] == [int(v) for v in ref[:4]]
    assert st["avgW"] == ref[4] and st["avgDeg"] == ref[5] and st["hScale"] == ref[6]


def test_genRMAT_reproduces_the_reference(oracle, gold):
    n, s, d, w = oracle.gen_rmat_ref(10, 8, 1000, 2026)
    row, col, wt, st = oracle.build_csr(n, s, d, w)
    assert np.array_equal(row, gold["rmat_row"])
    assert np.array_equal(col, gold["rmat_col"])
    assert np.array_equal(wt, gold["rmat_w"])


def test_buildCSR_edge_cases_match_the_reference(oracle, gold):
    # self loops dropped, w = 0 clamped to 1, duplicates kept, rows sorted by (w, dst)
    row, col, wt, st = oracle.build_csr(50, gold["build_in_src"], gold["build_in_dst"], gold["build_in_w"],
                                        gold["build_in_x"], gold["build_in_y"])
    assert np.array_equal(row, gold["build_row"])
    assert np.array_equal(col, gold["build_col"])
    assert np.array_equal(wt, gold["build_w"])
    assert st["hScale"] == gold["build_stats"][6]


def test_dijkstra_matches_the_reference_dist_and_parent(oracle, gold):
    g = graph(gold["road_row"], gold["road_col"], gold["road_w"])
    for i, s in enumerate(gold["road_srcs"]):
        d, p, _, _ = oracle.dijkstra(g, int(s))
        assert np.array_equal(d, gold["road_dist"][i])
        assert np.array_equal(p, gold["road_parent"][i])  # same heap order, same first relaxer
    g = graph(gold["rmat_row"], gold["rmat_col"], gold["rmat_w"])
    for i, s in enumerate(gold["rmat_srcs"]):
        d, p, _, _ = oracle.dijkstra(g, int(s))
        assert np.array_equal(d, gold["rmat_dist"][i])
        assert np.array_equal(p, gold["rmat_parent"][i])


def test_astar_matches_the_reference(oracle, gold):
    g = graph(gold["road_row"], gold["road_col"], gold["road_w"], gold["road_x"], gold["road_y"],
              float(gold["road_stats"][6]))
    off = 0
    for (s, t), dd, ln in zip(gold["road_astar_pairs"], gold["road_astar_dist"], gold["road_astar_len"]):
        d, path, _, _ = oracle.astar(g, int(s), int(t))
        assert d == dd
        assert path == gold["road_astar_paths"][off:off + ln].tolist()
        off += ln


def test_heuristic_matches_the_reference(oracle, gold):
    got = [oracle.heuristic(*map(float, p)) for p in gold["heur_in"]]
    assert got == gold["heur_out"].tolist()


def test_min_parent_is_the_smallest_tight_predecessor(oracle, gold):
    g = graph(gold["rmat_row"], gold["rmat_col"], gold["rmat_w"])
    s = int(gold["rmat_srcs"][0])
    d = gold["rmat_dist"][0]
    p = oracle.min_parent(g, d, s)
    row, col, w = g.row_offsets, g.col_indices, g.weights
    best = np.full(len(d), 0xFFFFFFFF, np.uint64)
    for u in range(len(d)):
        if d[u] == 0xFFFFFFFF:
            continue
        for k in range(row[u], row[u + 1]):
            v = col[k]
            if v != s and int(d[u]) + int(w[k]) == int(d[v]):
                best[v] = min(best[v], u)
    assert np.array_equal(p.astype(np.uint64), best)
    rep = oracle.verify_sssp(g, s, d, d, p, 64, 1)
    assert rep["errors"] == 0 and rep["treeChecked"] > 0


def test_verify_catches_a_planted_error(oracle, gold):
    # a mistake planted in a copy of the oracle's own output must be reported
    g = graph(gold["road_row"], gold["road_col"], gold["road_w"])
    s = int(gold["road_srcs"][0])
    d = gold["road_dist"][0].copy()
    p = gold["road_parent"][0].copy()
    v = int(np.flatnonzero(d != 0xFFFFFFFF)[5])
    bad = d.copy()
    bad[v] += 1
    assert oracle.verify_sssp(g, s, d, bad, p, 16, 0)["distMismatch"] == 1
    badp = p.copy()
    badp[v] = s if p[v] != s else (s + 1) % len(d)
    assert oracle.verify_sssp(g, s, d, d, badp, 16, 0)["treeErrors"] >= 1


@pytest.mark.slow
def test_reference_log_statistics(oracle):
    # results/colab_T4/logs/verify_grid_1e6.txt:7-10 and bench_rmat.txt:75-77 of the reference
    n, s, d, w, x, y = oracle.gen_grid_road(1000, 1000, 2026)
    _, _, _, st = oracle.build_csr(n, s, d, w, x, y)
    assert st["m"] == 4008120 and st["minW"] == 51 and st["maxW"] == 380 and st["maxDeg"] == 8
    assert round(st["avgW"], 1) == 155.9 and abs(st["hScale"] - 0.991796) < 5e-7
    n, s, d, w = oracle.gen_rmat_ref(20, 8, 1000, 2026)
    _, _, _, st = oracle.build_csr(n, s, d, w)
    assert st["m"] == 16084984 and st["maxDeg"] == 39665
    assert round(st["avgW"], 1) == 500.6
