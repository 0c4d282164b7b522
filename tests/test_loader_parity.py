"""Loader parity with the reference (CPU only).

The same DIMACS (.gr + .co), SNAP edge-list and PFCSR001 files are read by the
reference's own loaders (loadDIMACS / loadSNAP / loadBinary of src/graph.cpp,
compiled into oracle/_ref/libpfref.so, each edge list through its buildCSR) and by
this library's pfg_graph_load_*; the CSR arrays, coordinates, statistics and hScale
must be identical word for word. PFCSR001 is checked in both directions: a file
written here loads in the reference, and a file the reference's saveBinary writes
loads here. The files are written by this test (no dataset is needed).
"""
import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference CPU code not built (make -C oracle ref)")


def same_graph(ours, theirs, what):
    row, col, w, x, y, st = theirs.arrays()
    assert np.array_equal(ours.row_offsets, row), what
    assert np.array_equal(ours.col_indices, col), what
    assert np.array_equal(ours.weights, w), what
    if x is None:
        assert ours.x is None, what
    else:
        assert np.array_equal(ours.x, x) and np.array_equal(ours.y, y), what
    assert (ours.m, ours.minW, ours.maxW, ours.maxDeg) == (st["m"], st["minW"], st["maxW"], st["maxDeg"]), what
    # statistics and the heuristic scale are summed in the same order: equal to the bit
    assert ours.avgW == st["avgW"] and ours.avgDeg == st["avgDeg"], what
    assert ours.hScale == st["hScale"], what


def write_dimacs(tmp_path, n=300, m=1500, seed=3, comments=True):
    rng = np.random.default_rng(seed)
    gr = tmp_path / "g.gr"
    co = tmp_path / "g.co"
    src = rng.integers(1, n + 1, m)
    dst = rng.integers(1, n + 1, m)
    w = rng.integers(1, 5000, m)
    lines = []
    if comments:
        lines += ["c synthetic road network for the loader parity test", "c"]
    lines.append(f"p sp {n} {m}")
    lines += [f"a {a} {b} {c}" for a, b, c in zip(src, dst, w)]  # self loops and duplicates included
    gr.write_text("\n".join(lines) + "\n")
    xs = rng.integers(-74_000_000, -73_000_000, n)
    ys = rng.integers(40_000_000, 41_000_000, n)
    cl = ["c coordinates", f"p aux sp co {n}"] + [f"v {i + 1} {x} {y}" for i, (x, y) in enumerate(zip(xs, ys))]
    co.write_text("\n".join(cl) + "\n")
    return gr, co


def test_dimacs_with_coordinates(tmp_path):
    gr, co = write_dimacs(tmp_path)
    same_graph(pf.load_dimacs(str(gr), str(co)), O.ref_load_dimacs(gr, co), "dimacs .gr + .co")


def test_dimacs_without_coordinates(tmp_path):
    gr, _ = write_dimacs(tmp_path, n=120, m=700, seed=9, comments=False)
    same_graph(pf.load_dimacs(str(gr)), O.ref_load_dimacs(gr), "dimacs .gr")


@pytest.mark.parametrize("symmetrize", [True, False])
@pytest.mark.parametrize("weighted", [True, False])
def test_snap_edge_list(tmp_path, symmetrize, weighted):
    rng = np.random.default_rng(11)
    n, m = 500, 3000
    ids = rng.permutation(10_000)[:n]  # sparse, unordered vertex ids
    a, b = ids[rng.integers(0, n, m)], ids[rng.integers(0, n, m)]
    path = tmp_path / "edges.txt"
    lines = ["# Directed graph (each unordered pair of nodes is saved once)", "# FromNodeId\tToNodeId"]
    if weighted:
        w = rng.integers(1, 900, m)
        lines += [f"{x}\t{y}\t{z}" for x, y, z in zip(a, b, w)]
    else:
        lines += [f"{x}\t{y}" for x, y in zip(a, b)]
    path.write_text("\n".join(lines) + "\n")
    ours = pf.load_snap(str(path), symmetrize=symmetrize, max_w=1000, seed=2026)
    same_graph(ours, O.ref_load_snap(path, symmetrize, 1000, 2026), ("snap", symmetrize, weighted))


def test_pfcsr001_written_here_loads_in_the_reference(tmp_path):
    for g in (pf.grid(40, 30, 2026), pf.rmat(10, 8, seed=4)):
        p = tmp_path / "g.bin"
        g.save_binary(str(p))
        same_graph(g, O.ref_load_binary(p), "PFCSR001 here -> reference")
        same_graph(pf.load_binary(str(p)), O.ref_load_binary(p), "PFCSR001 round trip")


def test_pfcsr001_written_by_the_reference_loads_here(tmp_path):
    for rg in (O.ref_gen_grid_road(25, 35, 2026), O.ref_gen_rmat(10, 8, 1000, 2026)):
        p = tmp_path / "ref.bin"
        assert rg.save_binary(p)
        same_graph(pf.load_binary(str(p)), rg, "PFCSR001 reference -> here")
        assert p.read_bytes()[:8] == b"PFCSR001"


def test_malformed_files_fail_in_both(tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTACSR!" + b"\0" * 64)
    assert O.ref_load_binary(bad) is None
    with pytest.raises(Exception):
        pf.load_binary(str(bad))
    missing = tmp_path / "missing.gr"
    assert O.ref_load_dimacs(missing) is None
    with pytest.raises(Exception):
        pf.load_dimacs(str(missing))
