"""pfg_sssp_noalloc: the entry point for callers that may not allocate device memory.

Such callers (a plugin that may only touch the buffers its host application
hands it, or a latency-critical loop that cannot pay for cudaMalloc) get the
same persistent Delta-stepping kernel as pfg_run, with the kernel's scratch in
a fixed device array inside the library. This test owns the device buffers
(allocated here with torch), calls the entry point through the C ABI twice in a
row, and checks every packed (dist, parent) word against the regular entry
point pfg_run on the same graph and sources: integers, so the tolerance is zero.
"""
import ctypes as C

import numpy as np
import pytest

import pathfinding_gpu_b200 as pf
from pathfinding_gpu_b200 import _native as N

pytestmark = pytest.mark.gpu

PFG_ERR_CAPACITY = 8
MAX_VERTICES = 65536


def _device_csr(torch, g):
    dev = torch.device("cuda", 0)
    row = torch.from_numpy(g.row_offsets.astype(np.int32)).to(dev)
    col = torch.from_numpy(g.col_indices.astype(np.int32)).to(dev)
    w = torch.from_numpy(g.weights.astype(np.int32)).to(dev)
    return row, col, w


def _call(lib, row, col, w, n, m, src, delta, out, status, stream):
    return lib.pfg_sssp_noalloc(C.c_void_p(row.data_ptr()), C.c_void_p(col.data_ptr()),
                                C.c_void_p(w.data_ptr()), n, m, src, delta,
                                C.c_void_p(out.data_ptr()), C.c_void_p(status.data_ptr()),
                                C.c_void_p(stream))


def test_noalloc_matches_pfg_run_on_two_calls():
    torch = pytest.importorskip("torch")
    lib = N.load()
    g = pf.grid(100, 100, 2026)
    solver = pf.GpuSolver(g, 1)
    delta = solver.autoDelta()
    row, col, w = _device_csr(torch, g)
    out = torch.empty(g.n, dtype=torch.int64, device="cuda")
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for src in (0, 4321):  # two calls in a row share the one scratch array
        out.fill_(-1)
        status.zero_()
        st = _call(lib, row, col, w, g.n, g.m, src, delta, out, status, stream)
        assert st == 0, lib.pfg_last_error().decode()
        torch.cuda.synchronize()
        assert int(status[0].item()) == 0, f"device status {status.tolist()}"
        got = out.cpu().numpy().view(np.uint64)
        _, _, ref = solver.run_state([src], pf.GpuOptions(delta=delta))
        assert np.array_equal(got, ref), f"source {src}: {np.flatnonzero(got != ref)[:5]}"
    solver.close()


def test_noalloc_rejects_graphs_beyond_the_scratch_limit():
    torch = pytest.importorskip("torch")
    lib = N.load()
    small = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.empty(16, dtype=torch.int64, device="cuda")
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    st = _call(lib, small, small, small, MAX_VERTICES + 1, 4, 0, 100, out, status,
               torch.cuda.current_stream().cuda_stream)
    assert st == PFG_ERR_CAPACITY
    assert b"exceeds the fixed scratch limit" in lib.pfg_last_error()
