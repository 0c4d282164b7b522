"""Batches of uneven SSSP instances in one persistent launch (C ABI: pfg_batch_*).

    b = GpuBatch([g_big, g_small_1, ...], max_states=..., max_instances=...)
    b.set_instances([(0, s0), (0, s1), (1, s2), ...])   # (graph index, source)
    stats, ms = b.run(GpuOptions())                       # one launch for all instances
    b.capture(GpuOptions()); stats, ms = b.replay()       # the same run from a CUDA graph
    dist, parent = b.instance_result(i)

Generalises the reference's multiSource (k*n + v indexing, src/gpu_sssp.cu:553-569)
to per-instance offsets so graphs of different sizes share one launch.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .graphs import CSRGraph
from .solver import GpuOptions, GpuStats, unpack


class GpuBatch:
    def __init__(self, graphs: Sequence[CSRGraph], max_states: Optional[int] = None,
                 max_instances: int = 1024, device: int = 0):
        self._lib = N.load()
        self.graphs = list(graphs)
        self._keep = []
        rows, cols, ws = [], [], []
        for g in self.graphs:
            r = np.ascontiguousarray(g.row_offsets, np.uint32)
            c = np.ascontiguousarray(g.col_indices if g.m else np.zeros(1, np.uint32), np.uint32)
            w = np.ascontiguousarray(g.weights if g.m else np.zeros(1, np.uint32), np.uint32)
            self._keep += [r, c, w]
            rows.append(N.ptr(r, N.u32))
            cols.append(N.ptr(c, N.u32))
            ws.append(N.ptr(w, N.u32))
        G = len(self.graphs)
        PA = C.POINTER(N.u32) * G
        ns = np.asarray([g.n for g in self.graphs], np.uint32)
        ms = np.asarray([g.m for g in self.graphs], np.uint32)
        if max_states is None:
            max_states = int(sum(g.n for g in self.graphs))
        h = C.c_void_p()
        N.check(self._lib.pfg_batch_create(G, PA(*rows), PA(*cols), PA(*ws), N.ptr(ns, N.u32),
                                           N.ptr(ms, N.u32), int(max_states), int(max_instances),
                                           int(device), C.byref(h)))
        self._h = h
        self.instances: List[Tuple[int, int]] = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pfg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_instances(self, instances: Sequence[Tuple[int, int]]) -> None:
        g = np.ascontiguousarray([a for a, _ in instances], np.uint32)
        s = np.ascontiguousarray([b for _, b in instances], np.uint32)
        N.check(self._lib.pfg_batch_set_instances(self._h, N.ptr(g, N.u32), N.ptr(s, N.u32), len(g)))
        self.instances = [(int(a), int(b)) for a, b in instances]

    def run(self, opt: Optional[GpuOptions] = None):
        c = (opt or GpuOptions()).to_c()
        st = N.PfgStats()
        ms = C.c_float()
        N.check(self._lib.pfg_batch_run(self._h, C.byref(c), C.byref(st), C.byref(ms)))
        return GpuStats.from_c(st), float(ms.value)

    def capture(self, opt: Optional[GpuOptions] = None) -> None:
        c = (opt or GpuOptions()).to_c()
        N.check(self._lib.pfg_batch_capture(self._h, C.byref(c)))

    def replay(self):
        st = N.PfgStats()
        ms = C.c_float()
        N.check(self._lib.pfg_batch_replay(self._h, C.byref(st), C.byref(ms)))
        return GpuStats.from_c(st), float(ms.value)

    def offset(self, inst: int) -> int:
        return int(self._lib.pfg_batch_instance_offset(self._h, inst))

    def num_states(self) -> int:
        return int(self._lib.pfg_batch_num_states(self._h))

    def stream(self) -> int:
        return self._lib.pfg_batch_stream(self._h)

    def device_bytes(self) -> int:
        return int(self._lib.pfg_batch_device_bytes(self._h))

    def state(self) -> np.ndarray:
        out = np.empty(self.num_states(), np.uint64)
        N.check(self._lib.pfg_batch_copy_state(self._h, 0, len(out), N.ptr(out, N.u64)))
        return out

    def instance_result(self, inst: int, state: Optional[np.ndarray] = None):
        a, b = self.offset(inst), self.offset(inst + 1)
        if state is None:
            out = np.empty(b - a, np.uint64)
            N.check(self._lib.pfg_batch_copy_state(self._h, a, b - a, N.ptr(out, N.u64)))
        else:
            out = state[a:b]
        return unpack(out)
