"""CSR construction on the GPU (pfg_graph_from_edges_gpu / pfg_csr_build_device):
row offsets, columns, weights and statistics identical word for word to the
host builder and to the oracle's restatement of the reference's buildCSR,
including rows in every sort tier (<= 32 arcs, <= 2048, hub rows merged)."""
import ctypes as C

import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import _native as N

pytestmark = pytest.mark.gpu


def arcs_of(g):
    deg = np.diff(g.row_offsets).astype(np.int64)
    src = np.repeat(np.arange(g.n, dtype=np.uint32), deg)
    return src, g.col_indices.copy(), g.weights.copy()


def check_same(oracle, n, src, dst, w, x=None, y=None):
    host = pf.buildCSR(n, src, dst, w, x, y)
    dev = pf.buildCSR(n, src, dst, w, x, y, device=0)
    assert np.array_equal(dev.row_offsets, host.row_offsets)
    assert np.array_equal(dev.col_indices, host.col_indices)
    assert np.array_equal(dev.weights, host.weights)
    for f in ("minW", "maxW", "maxDeg", "avgW", "avgDeg", "hScale"):
        assert getattr(dev, f) == getattr(host, f), f
    row, col, wt, st = oracle.build_csr(n, src, dst, w, x, y)
    assert np.array_equal(dev.row_offsets, row) and np.array_equal(dev.col_indices, col)
    assert np.array_equal(dev.weights, wt)
    assert dev.hScale == st["hScale"] and dev.avgW == st["avgW"]
    return dev


def test_random_arcs_self_loops_zero_weights_duplicates(oracle):
    rng = np.random.default_rng(1)
    n = 5000
    m = 60000
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    dst[:500] = src[:500]  # self loops are dropped
    w = rng.integers(0, 20, m).astype(np.uint32)  # zeros become 1, many ties
    src[-2000:] = src[:2000]
    dst[-2000:] = dst[:2000]  # duplicate arcs are kept
    x = rng.uniform(0, 100, n)
    y = rng.uniform(0, 100, n)
    g = check_same(oracle, n, src, dst, w, x, y)
    assert g.minW == 1


@pytest.mark.parametrize("lens", [[2, 31, 32, 33], [2047, 2048, 2049], [4096, 6000, 10000], [70000]])
def test_row_length_tiers(oracle, lens):
    rng = np.random.default_rng(sum(lens))
    n = 100000
    srcs, dsts = [], []
    for i, L in enumerate(lens):
        srcs.append(np.full(L, 7 + 11 * i, np.uint32))
        dsts.append(rng.integers(0, n, L).astype(np.uint32))
    src = np.concatenate(srcs)
    dst = np.concatenate(dsts)
    w = rng.integers(1, 50, len(src)).astype(np.uint32)
    perm = rng.permutation(len(src))
    check_same(oracle, n, src[perm], dst[perm], w[perm])


def test_generator_graphs_rebuilt(oracle):
    for g in (pf.grid(300, 300, 5), pf.road(256, seed=3), pf.rmat(14, 64, seed=4)):
        src, dst, w = arcs_of(g)
        perm = np.random.default_rng(0).permutation(len(src))
        dev = check_same(oracle, g.n, src[perm], dst[perm], w[perm], g.x, g.y)
        assert np.array_equal(dev.col_indices, g.col_indices)
        assert dev.hScale == g.hScale


def test_empty_and_isolated():
    g = pf.buildCSR(10, [], [], [], device=0)
    assert g.m == 0 and np.array_equal(g.row_offsets, np.zeros(11, np.uint32))
    g = pf.buildCSR(4, [1, 1, 2], [1, 3, 0], [5, 0, 2], device=0)
    assert g.m == 2 and list(g.row_offsets) == [0, 0, 1, 2, 2]


def test_out_of_range_endpoint_is_an_error():
    with pytest.raises(RuntimeError):
        pf.buildCSR(4, [0, 9], [1, 2], [1, 1], device=0)


def test_device_pointer_entry_point():
    torch = pytest.importorskip("torch")
    g = pf.grid(64, 64, 9)
    src, dst, w = arcs_of(g)
    perm = np.random.default_rng(2).permutation(len(src))
    dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).astype(dt)).cuda()
    d_src, d_dst, d_w = dev(src[perm], np.int32), dev(dst[perm], np.int32), dev(w[perm], np.int32)
    d_x, d_y = dev(g.x, np.float64), dev(g.y, np.float64)
    row = torch.empty(g.n + 1, dtype=torch.int32, device="cuda")
    col = torch.empty(len(src), dtype=torch.int32, device="cuda")
    wo = torch.empty(len(src), dtype=torch.int32, device="cuda")
    info = N.PfgGraphInfo()
    vp = lambda t: C.c_void_p(t.data_ptr())
    N.check(N.load().pfg_csr_build_device(g.n, len(src), vp(d_src), vp(d_dst), vp(d_w), vp(d_x), vp(d_y),
                                          vp(row), vp(col), vp(wo), C.byref(info), 0, None))
    assert info.m == g.m and info.h_scale == g.hScale and info.max_deg == g.maxDeg
    assert np.array_equal(row.cpu().numpy().view(np.uint32), g.row_offsets)
    assert np.array_equal(col.cpu().numpy().view(np.uint32), g.col_indices)
    assert np.array_equal(wo.cpu().numpy().view(np.uint32), g.weights)
