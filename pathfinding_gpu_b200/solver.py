"""Python mirror of the reference's GpuSolver interface (include/gpu_sssp.h:10-120).

Same names, argument meaning and error behaviour as the reference's C++ class:
`GpuSolver(g, maxBatch)`, `sssp(src, opt, copyBack)`, `astar(src, dst, opt)`,
`multiSource(srcs, opt, distOut)`, `uploadMs()`, `deviceBytes()`, `autoDelta()`;
invalid batches, sources and targets raise RuntimeError (the reference throws
std::runtime_error, src/gpu_sssp.cu:463-465). Everything runs through the C ABI
of libpfg_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from enum import IntEnum
from typing import List, Optional

import numpy as np

from . import _native as N
from .graphs import CSRGraph

INF_DIST = 0xFFFFFFFF
NO_PARENT = 0xFFFFFFFF


class GpuAlgo(IntEnum):
    NaiveRelax = 0
    Frontier = 1
    DeltaStep = 2


class Mapping(IntEnum):
    Thread = 0
    Warp = 1
    Hybrid = 2


class AtomicMode(IntEnum):
    MinRBA = 0
    CasRBA = 1
    MinNoCheck = 2


class Compaction(IntEnum):
    WarpAtomic = 0
    PrefixScan = 1


class Policy(IntEnum):
    Fixed = 0
    Learned = 1


class Schedule(IntEnum):
    """How a Delta-stepping bucket is worked off (pfg_schedule in include/pfg.h)."""
    Auto = 0    # Instance from 96 sources where it applies, else Async for Delta-stepping; Rounds otherwise
    Rounds = 1  # relaxation rounds separated by grid barriers (the reference's loop)
    Async = 2   # one drain per bucket through CTA claimed lists and a ring queue
    Warp = 3    # Async, the drain worked by independent warps (Hybrid mapping)
    Instance = 4  # Async with a bucket window per instance of a multi-source run (falls back to Async)


@dataclass
class GpuOptions:
    algo: GpuAlgo = GpuAlgo.DeltaStep
    mapping: Mapping = Mapping.Hybrid
    atomic: AtomicMode = AtomicMode.MinRBA
    delta: int = 0
    blockSize: int = 256
    syncEvery: int = 8
    compaction: Compaction = Compaction.WarpAtomic
    policy: Policy = Policy.Fixed
    eager: int = -1  # Hybrid mapping: eager sub-rounds per grid round (-1 engine default, 0 off)
    blocksPerSM: int = 0  # CTAs of the persistent kernel per SM (0: engine default)
    schedule: Schedule = Schedule.Auto

    def to_c(self) -> N.PfgOptions:
        return N.PfgOptions(int(self.algo), int(self.mapping), int(self.atomic), int(self.delta),
                            int(self.blockSize), int(self.syncEvery), int(self.compaction),
                            int(self.policy), int(self.eager), int(self.blocksPerSM), int(self.schedule))


@dataclass
class GpuStats:
    edgesScanned: int = 0
    atomicsIssued: int = 0
    updates: int = 0
    pushes: int = 0
    iterations: int = 0
    hostSyncs: int = 0
    launches: int = 0
    buckets: int = 0
    delta: int = 0
    rounds: int = 0

    @staticmethod
    def from_c(s: N.PfgStats) -> "GpuStats":
        return GpuStats(s.edges_scanned, s.atomics_issued, s.updates, s.pushes, s.iterations,
                        s.host_syncs, s.launches, s.buckets, s.delta, s.rounds)


@dataclass
class GpuRunResult:
    ms: float = 0.0
    stats: GpuStats = field(default_factory=GpuStats)
    dist: Optional[np.ndarray] = None
    parent: Optional[np.ndarray] = None
    targetDist: int = INF_DIST
    path: List[int] = field(default_factory=list)


def unpack(state: np.ndarray):
    """Packed (dist << 32) | parent words -> (dist, parent) uint32 arrays."""
    state = np.asarray(state, np.uint64)
    return (state >> np.uint64(32)).astype(np.uint32), (state & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def reconstruct_path(parent: np.ndarray, src: int, dst: int) -> List[int]:
    """Parent chain dst -> src reversed; [] when broken (reference reconstructPath)."""
    n = len(parent)
    if dst >= n:
        return []
    path, v = [], int(dst)
    for _ in range(n + 1):
        path.append(v)
        if v == src:
            return path[::-1]
        v = int(parent[v])
        if v == NO_PARENT or v >= n:
            break
    return []


class GpuSolver:
    """Holds the CSR graph and all working buffers on one GPU (allocated once)."""

    def __init__(self, g: CSRGraph, maxBatch: int = 1, device: int = 0):
        self._lib = N.load()
        self.g = g
        self.n = g.n
        self._row = np.ascontiguousarray(g.row_offsets, np.uint32)
        self._col = np.ascontiguousarray(g.col_indices, np.uint32)
        self._w = np.ascontiguousarray(g.weights, np.uint32)
        x = None if g.x is None else np.ascontiguousarray(g.x, np.float64)
        y = None if g.y is None else np.ascontiguousarray(g.y, np.float64)
        h = C.c_void_p()
        N.check(self._lib.pfg_create_on_device(
            N.ptr(self._row, N.u32), N.ptr(self._col, N.u32), N.ptr(self._w, N.u32),
            N.ptr(x, N.f64), N.ptr(y, N.f64), g.n, g.m, float(g.hScale), float(g.avgW),
            float(g.avgDeg), max(1, int(maxBatch)), int(device), C.byref(h)))
        self._h = h
        self.maxBatch = max(1, int(maxBatch))

    # ---- life cycle ----
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pfg_destroy(self._h)
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

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise RuntimeError("solver is closed")
        return self._h

    # ---- accessors ----
    def uploadMs(self) -> float:
        return self._lib.pfg_upload_ms(self.handle)

    def deviceBytes(self) -> int:
        return self._lib.pfg_device_bytes(self.handle)

    def autoDelta(self) -> int:
        return self._lib.pfg_auto_delta(self.handle)

    def stream(self) -> int:
        return self._lib.pfg_stream(self.handle)

    # ---- runs ----
    def run_state(self, srcs, opt: Optional[GpuOptions] = None, astar: bool = False, dst: int = 0,
                  copy: bool = True, out: Optional[np.ndarray] = None):
        """One run; returns (GpuStats, ms, packed state of k*n words or None)."""
        srcs = np.ascontiguousarray(np.atleast_1d(srcs), np.uint32)
        k = len(srcs)
        opt = opt or GpuOptions()
        c = opt.to_c()
        st = N.PfgStats()
        ms = C.c_float(0.0)
        state = None
        if copy:
            state = out if out is not None else np.empty(k * self.n, np.uint64)
        N.check(self._lib.pfg_run(self.handle, N.ptr(srcs, N.u32), k, 1 if astar else 0, int(dst),
                                  C.byref(c), C.byref(st), N.ptr(state, N.u64), C.byref(ms)))
        return GpuStats.from_c(st), float(ms.value), state

    def sssp(self, src: int, opt: Optional[GpuOptions] = None, copyBack: bool = True) -> GpuRunResult:
        stats, ms, state = self.run_state([src], opt, copy=copyBack)
        r = GpuRunResult(ms=ms, stats=stats)
        if state is not None:
            r.dist, r.parent = unpack(state)
        return r

    def astar(self, src: int, dst: int, opt: Optional[GpuOptions] = None) -> GpuRunResult:
        stats, ms, state = self.run_state([src], opt, astar=True, dst=dst, copy=True)
        r = GpuRunResult(ms=ms, stats=stats)
        dist, parent = unpack(state)
        r.targetDist = int(dist[dst])
        if r.targetDist != INF_DIST:
            r.path = reconstruct_path(parent, src, dst)
        return r

    def astar_device_path(self, src: int, dst: int, opt: Optional[GpuOptions] = None,
                          cap: Optional[int] = None) -> GpuRunResult:
        """A* whose path is rebuilt on the device; only the path crosses PCIe."""
        stats, ms, _ = self.run_state([src], opt, astar=True, dst=dst, copy=False)
        r = GpuRunResult(ms=ms, stats=stats)
        d = np.empty(1, np.uint64)
        N.check(self._lib.pfg_copy_state(self.handle, int(dst), 1, N.ptr(d, N.u64)))
        r.targetDist = int(d[0] >> np.uint64(32))
        if r.targetDist != INF_DIST:
            r.path = self.extract_path(0, src, dst, cap)
        return r

    def extract_path(self, inst: int, src: int, dst: int, cap: Optional[int] = None) -> List[int]:
        cap = self.n + 1 if cap is None else int(cap)
        buf = np.empty(cap, np.uint32)
        ln = C.c_uint32(0)
        N.check(self._lib.pfg_extract_path(self.handle, int(inst), int(src), int(dst),
                                           N.ptr(buf, N.u32), cap, C.byref(ln)))
        return buf[: ln.value].tolist()

    def multiSource(self, srcs, opt: Optional[GpuOptions] = None,
                    distOut: Optional[list] = None) -> GpuRunResult:
        srcs = np.ascontiguousarray(srcs, np.uint32)
        k = len(srcs)
        stats, ms, _ = self.run_state(srcs, opt, copy=False)
        r = GpuRunResult(ms=ms, stats=stats)
        if distOut is not None:
            dist = self.copy_dist(0, k * self.n)
            distOut.clear()
            distOut.extend(dist.reshape(k, self.n))
        return r

    def run_dist_async(self, srcs, out: np.ndarray, opt: Optional[GpuOptions] = None) -> GpuStats:
        """Streamed multiSource: enqueues a run of `srcs` whose distances go to `out`
        (k*n uint32, pinned for an asynchronous copy; valid until dist_wait) and starts
        copying the previous streamed run's distances while this one computes.
        Returns the previous run's statistics."""
        srcs = np.ascontiguousarray(np.atleast_1d(srcs), np.uint32)
        assert out.dtype == np.uint32 and out.flags.c_contiguous and out.size >= len(srcs) * self.n
        c = (opt or GpuOptions()).to_c()
        st = N.PfgStats()
        N.check(self._lib.pfg_run_dist_async(self.handle, N.ptr(srcs, N.u32), len(srcs), C.byref(c),
                                             N.ptr(out, N.u32), C.byref(st)))
        return GpuStats.from_c(st)

    def dist_wait(self) -> GpuStats:
        """Completes the stream: the last run and every distance copy."""
        st = N.PfgStats()
        N.check(self._lib.pfg_dist_wait(self.handle, C.byref(st)))
        return GpuStats.from_c(st)

    def copy_dist(self, first: int, count: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Distances of state words [first, first+count) of the last run (split from
        the packed words on the device; 4 bytes per word cross PCIe)."""
        if out is None:
            out = np.empty(count, np.uint32)
        assert out.dtype == np.uint32 and out.flags.c_contiguous and out.size >= count
        N.check(self._lib.pfg_copy_dist(self.handle, int(first), int(count), N.ptr(out, N.u32)))
        return out[:count]

    def set_policy(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, np.float32)
        N.check(self._lib.pfg_set_policy(self.handle, N.ptr(params, N.f32), params.size))


def device_info(dev: int = 0) -> N.PfgDeviceInfo:
    info = N.PfgDeviceInfo()
    N.check(N.load().pfg_query_device(dev, C.byref(info)))
    return info
