"""pfg_sssp_noalloc: the entry point for callers that may not allocate device memory.

Such callers (a plugin that may only touch the buffers its host application
hands it, or a latency-critical loop that cannot pay for cudaMalloc) get the
same persistent Delta-stepping kernel as pfg_run, with the kernel's scratch in
a fixed device array inside the library. These tests own the device buffers
(allocated here with torch), call the entry point through the C ABI, and check
every packed (dist, parent) word against the regular entry point pfg_run on the
same graph and source, and against the oracle: integers, so the tolerance is
zero. They also cover the size limits of the fixed array and the device-side
checks of the caller's CSR (every malformed input below is turned into an error
status by those checks before any relaxation; no access leaves the buffers).
"""
import ctypes as C

import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import _native as N

pytestmark = pytest.mark.gpu

PFG_ERR_INVALID_GRAPH = 2
PFG_ERR_CAPACITY = 8
MAX_VERTICES = 65536
MAX_ARCS = 655360


def _device_csr(torch, row, col, w):
    dev = torch.device("cuda", 0)
    as_t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).to(dev)
    return as_t(row), as_t(col if len(col) else np.zeros(1, np.uint32)), as_t(w if len(w) else np.ones(1, np.uint32))


def _call(lib, row, col, w, n, m, src, delta, out, status, stream):
    return lib.pfg_sssp_noalloc(C.c_void_p(row.data_ptr()), C.c_void_p(col.data_ptr()),
                                C.c_void_p(w.data_ptr()), n, m, src, delta,
                                C.c_void_p(out.data_ptr()), C.c_void_p(status.data_ptr()),
                                C.c_void_p(stream))


def _run(torch, lib, row, col, w, n, m, src, delta):
    """One call on device copies of the arrays; returns (host state words, status words)."""
    d_row, d_col, d_w = _device_csr(torch, row, col, w)
    out = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    status = torch.full((4,), -7, dtype=torch.int32, device="cuda")
    st = _call(lib, d_row, d_col, d_w, n, m, src, delta, out, status, torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.pfg_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64).copy(), status.cpu().numpy().view(np.uint32).copy()


def _check_against_run_and_oracle(torch, lib, oracle, g, srcs):
    solver = pf.GpuSolver(g, 1)
    delta = solver.autoDelta()
    for src in srcs:  # consecutive calls share the one scratch array
        got, status = _run(torch, lib, g.row_offsets, g.col_indices, g.weights, g.n, g.m, src, delta)
        assert status[0] == 0, f"device status {status.tolist()}"
        _, _, ref = solver.run_state([src], pf.GpuOptions(delta=delta))
        assert np.array_equal(got, ref), f"source {src}: {np.flatnonzero(got != ref)[:5]}"
        d_ref, p_can = oracle.sssp_canonical(g, src)
        dist, parent = pf.unpack(got)
        assert np.array_equal(dist, d_ref) and np.array_equal(parent, p_can), f"source {src} vs the oracle"
    solver.close()


def test_noalloc_matches_pfg_run_on_two_calls(oracle):
    torch = pytest.importorskip("torch")
    lib = N.load()
    g = pf.grid(100, 100, 2026)
    _check_against_run_and_oracle(torch, lib, oracle, g, (0, 4321))


def test_noalloc_power_law_graph(oracle):
    # a skewed R-MAT graph: long rows are relaxed by the CTA that holds them (no hub records here)
    torch = pytest.importorskip("torch")
    lib = N.load()
    g = pf.rmat(14, 16, seed=2026)
    assert g.n <= MAX_VERTICES and g.m + 3 * g.n <= MAX_ARCS
    _check_against_run_and_oracle(torch, lib, oracle, g, pf.pick_sources(g, 2, 5).tolist())


def test_noalloc_at_the_scratch_limits(oracle):
    # n = 65,536 vertices and m + 3n just under the padded-arc limit: the last
    # offsets of every scratch region are used
    torch = pytest.importorskip("torch")
    lib = N.load()
    n = MAX_VERTICES
    rng = np.random.default_rng(7)
    m_target = MAX_ARCS - 3 * n - 8
    # a ring (every vertex reachable) plus random arcs
    src = np.concatenate([np.arange(n), rng.integers(0, n, m_target - n)]).astype(np.uint32)
    dst = np.concatenate([(np.arange(n) + 1) % n, rng.integers(0, n, m_target - n)]).astype(np.uint32)
    w = rng.integers(1, 1000, m_target).astype(np.uint32)
    g = pf.buildCSR(n, src, dst, w)
    assert g.n == n and g.m + 3 * g.n <= MAX_ARCS and g.m + 3 * g.n > MAX_ARCS - 3 * n // 2
    _check_against_run_and_oracle(torch, lib, oracle, g, (0, n - 1))


def test_noalloc_single_vertex():
    torch = pytest.importorskip("torch")
    lib = N.load()
    got, status = _run(torch, lib, np.zeros(2, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32),
                       1, 0, 0, 100)
    assert status[0] == 0
    assert got[0] == np.uint64(pf.NO_PARENT)  # dist 0, no parent


def test_noalloc_rejects_graphs_beyond_the_scratch_limit():
    torch = pytest.importorskip("torch")
    lib = N.load()
    small = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _call(lib, small, small, small, MAX_VERTICES + 1, 4, 0, 100, out, status, stream)
    assert st == PFG_ERR_CAPACITY
    assert b"exceeds the fixed scratch limit" in lib.pfg_last_error()
    # m + 3n one over the padded-arc limit (checked on the host, nothing launched)
    n = 1000
    st = _call(lib, small, small, small, n, MAX_ARCS - 3 * n + 1, 0, 100, out, status, stream)
    assert st == PFG_ERR_CAPACITY
    assert b"padded arcs" in lib.pfg_last_error()


@pytest.mark.parametrize("case", ["column", "weight", "order", "row_end", "decreasing"])
def test_noalloc_device_side_csr_checks(case):
    # the host cannot read the caller's device arrays without waiting: malformed
    # CSRs are caught on the device, reported in the status words, and nothing is relaxed
    torch = pytest.importorskip("torch")
    lib = N.load()
    g = pf.grid(20, 20, 3)
    row, col, w = g.row_offsets.copy(), g.col_indices.copy(), g.weights.copy()
    m = g.m
    if case == "column":
        col[17] = g.n + 5
        bit = 4
    elif case == "weight":
        w[3] = 0
        bit = 8
    elif case == "order":
        b = row[42]
        w[b], w[b + 1] = w[b + 1] + 10, w[b]  # first arc heavier than the second
        bit = 16
    elif case == "row_end":
        m = g.m - 1  # row_offsets[n] != m
        bit = 1
    else:
        row[5] = row[6] + 1  # a decreasing offset
        bit = 1
    got, status = _run(torch, lib, row, col, w, g.n, m, 0, 100)
    want = PFG_ERR_INVALID_GRAPH
    assert status[0] == want and (status[1] & bit), status.tolist()
    assert np.all(got == np.uint64(0xFFFFFFFFFFFFFFFF)), "a rejected graph must not be relaxed"
    # a later valid call on the same scratch is exact again
    good, status = _run(torch, lib, g.row_offsets, g.col_indices, g.weights, g.n, g.m, 0, 100)
    assert status[0] == 0
    with pf.GpuSolver(g, 1) as s:
        _, _, ref = s.run_state([0], pf.GpuOptions(delta=100))
    assert np.array_equal(good, ref)
