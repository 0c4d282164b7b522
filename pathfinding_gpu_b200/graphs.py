"""CSR graphs and the seeded synthetic workloads (host side, native code in pfg_graphs.cpp).

`CSRGraph` mirrors the reference's struct (include/graph.h:31-48): row_offsets /
col_indices / weights as uint32 arrays with every row sorted by (w, dst),
optional float64 coordinates, and the statistics n, m, minW, maxW, maxDeg,
avgW, avgDeg, hScale.

Workloads (all SplitMix64-seeded, default seed 2026):
  grid(side)              side x side grid, 4-neighbour arcs both ways, w = llround(100 U[1,1.5))
  rmat(20, 16)            directed R-MAT (.57,.19,.19,.05), self loops dropped, duplicates keep
                          the lightest copy, w uniform in [1, 255]
  road(2048)              grid with 10% of neighbour pairs removed and 1% of vertices given a
                          bidirectional shortcut within 64 cells, w = ceil(1.2 * 100 * Euclid)
  grid_batch(256)         independent grids with sides log-uniform in [32, 316]
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _native as N

DEFAULT_SEED = 2026


@dataclass
class CSRGraph:
    row_offsets: np.ndarray
    col_indices: np.ndarray
    weights: np.ndarray
    x: Optional[np.ndarray] = None
    y: Optional[np.ndarray] = None
    name: str = ""
    hScale: float = 0.0
    minW: int = 0
    maxW: int = 0
    maxDeg: int = 0
    avgW: float = 0.0
    avgDeg: float = 0.0

    @property
    def n(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    @property
    def m(self) -> int:
        return int(self.col_indices.shape[0])

    def hasCoords(self) -> bool:
        return self.x is not None

    def degree(self, u: int) -> int:
        return int(self.row_offsets[u + 1] - self.row_offsets[u])

    def bytesCSR(self) -> int:
        return (self.n + 1) * 4 + self.m * 8

    # ---- native handle round trip ----
    @staticmethod
    def _from_handle(h: C.c_void_p, name: str = "") -> "CSRGraph":
        lib = N.load()
        info = N.PfgGraphInfo()
        try:
            N.check(lib.pfg_graph_get_info(h, C.byref(info)))
            n, m = info.n, info.m
            row = np.ctypeslib.as_array(lib.pfg_graph_row_offsets(h), shape=(n + 1,)).copy()
            col = (np.ctypeslib.as_array(lib.pfg_graph_col_indices(h), shape=(m,)).copy() if m
                   else np.zeros(0, np.uint32))
            w = (np.ctypeslib.as_array(lib.pfg_graph_weights(h), shape=(m,)).copy() if m
                 else np.zeros(0, np.uint32))
            x = y = None
            if info.has_xy:
                x = np.ctypeslib.as_array(lib.pfg_graph_x(h), shape=(n,)).copy()
                y = np.ctypeslib.as_array(lib.pfg_graph_y(h), shape=(n,)).copy()
        finally:
            lib.pfg_graph_free(h)
        return CSRGraph(row, col, w, x, y, name, info.h_scale, info.min_w, info.max_w, info.max_deg,
                        info.avg_w, info.avg_deg)

    def _to_handle(self) -> C.c_void_p:
        lib = N.load()
        n = self.n
        src = np.repeat(np.arange(n, dtype=np.uint32), np.diff(self.row_offsets).astype(np.int64))
        col = np.ascontiguousarray(self.col_indices, np.uint32)
        w = np.ascontiguousarray(self.weights, np.uint32)
        x = None if self.x is None else np.ascontiguousarray(self.x, np.float64)
        y = None if self.y is None else np.ascontiguousarray(self.y, np.float64)
        h = C.c_void_p()
        N.check(lib.pfg_graph_from_edges(n, self.m, N.ptr(src, N.u32), N.ptr(col, N.u32),
                                         N.ptr(w, N.u32), N.ptr(x, N.f64), N.ptr(y, N.f64),
                                         C.byref(h)))
        return h

    def save_binary(self, path: str) -> None:
        """Writes the reference's PFCSR001 binary cache (src/graph.cpp:320-336)."""
        lib = N.load()
        h = self._to_handle()
        try:
            N.check(lib.pfg_graph_save_binary(h, str(path).encode()))
        finally:
            lib.pfg_graph_free(h)


def _gen(fn_name: str, *args, name: str = "") -> CSRGraph:
    lib = N.load()
    h = C.c_void_p()
    N.check(getattr(lib, fn_name)(*args, C.byref(h)))
    return CSRGraph._from_handle(h, name)


def buildCSR(n: int, src, dst, w, x=None, y=None, name: str = "", device: Optional[int] = None) -> CSRGraph:
    """CSR from an arc list (reference buildCSR, src/graph.cpp:23-104).

    device=None builds on the host; device=d sorts and counts on GPU d
    (pfg_graph_from_edges_gpu), with an identical result."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = np.ascontiguousarray(w, np.uint32)
    x = None if x is None else np.ascontiguousarray(x, np.float64)
    y = None if y is None else np.ascontiguousarray(y, np.float64)
    if not (len(src) == len(dst) == len(w)):
        raise ValueError("src, dst and w must have the same length")
    if device is not None:
        return _gen("pfg_graph_from_edges_gpu", n, len(src), N.ptr(src, N.u32), N.ptr(dst, N.u32),
                    N.ptr(w, N.u32), N.ptr(x, N.f64), N.ptr(y, N.f64), int(device), name=name)
    return _gen("pfg_graph_from_edges", n, len(src), N.ptr(src, N.u32), N.ptr(dst, N.u32),
                N.ptr(w, N.u32), N.ptr(x, N.f64), N.ptr(y, N.f64), name=name)


def grid(rows: int, cols: Optional[int] = None, seed: int = DEFAULT_SEED) -> CSRGraph:
    cols = rows if cols is None else cols
    return _gen("pfg_graph_gen_grid", rows, cols, seed, name=f"grid_{rows}x{cols}")


def rmat(scale: int = 20, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         w_lo: int = 1, w_hi: int = 255, seed: int = DEFAULT_SEED) -> CSRGraph:
    return _gen("pfg_graph_gen_rmat", scale, edge_factor, a, b, c, w_lo, w_hi, seed,
                name=f"rmat_s{scale}_ef{edge_factor}")


def road(side: int = 2048, removal: float = 0.10, shortcut: float = 0.01, radius: int = 64,
         factor: float = 1.2, seed: int = DEFAULT_SEED) -> CSRGraph:
    return _gen("pfg_graph_gen_road", side, removal, shortcut, radius, factor, seed,
                name=f"road_{side}x{side}")


def grid_batch_sides(count: int = 256, lo: int = 32, hi: int = 316, seed: int = DEFAULT_SEED) -> list:
    """Side lengths drawn log-uniform in [lo, hi] from a SplitMix64 stream."""
    rng = SplitMix64(seed)
    return [int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(count)]


def grid_batch(count: int = 256, lo: int = 32, hi: int = 316, seed: int = DEFAULT_SEED) -> list:
    sides = grid_batch_sides(count, lo, hi, seed)
    return [grid(s, s, seed + 1 + i) for i, s in enumerate(sides)]


def union(parts: Sequence[CSRGraph]) -> tuple:
    """Disjoint union; returns (graph, vertex offset of each part)."""
    lib = N.load()
    handles = [p._to_handle() for p in parts]
    try:
        arr = (C.c_void_p * len(handles))(*handles)
        h = C.c_void_p()
        N.check(lib.pfg_graph_union(arr, len(handles), C.byref(h)))
    finally:
        for hh in handles:
            lib.pfg_graph_free(hh)
    g = CSRGraph._from_handle(h, f"union_{len(parts)}")
    offs = np.cumsum([0] + [p.n for p in parts[:-1]]).astype(np.int64)
    return g, offs


def load_dimacs(gr_path: str, co_path: Optional[str] = None) -> CSRGraph:
    return _gen("pfg_graph_load_dimacs", str(gr_path).encode(),
                None if co_path is None else str(co_path).encode())


def load_snap(path: str, symmetrize: bool = True, max_w: int = 1000, seed: int = DEFAULT_SEED) -> CSRGraph:
    return _gen("pfg_graph_load_snap", str(path).encode(), 1 if symmetrize else 0, max_w, seed)


def load_binary(path: str) -> CSRGraph:
    return _gen("pfg_graph_load_binary", str(path).encode())


def pick_sources(g: CSRGraph, count: int, seed: int) -> np.ndarray:
    """Vertices with out-degree > 0 (reference pickSources, src/graph.cpp:369-378)."""
    rng = SplitMix64(seed)
    deg = np.diff(g.row_offsets)
    out = []
    tries = 0
    while len(out) < count and tries < count * 1000 + 1000:
        v = rng.below(g.n)
        if deg[v] > 0:
            out.append(v)
        tries += 1
    out += [0] * (count - len(out))
    return np.asarray(out, np.uint32)


def uniform_vertices(n: int, count: int, seed: int) -> np.ndarray:
    rng = SplitMix64(seed)
    return np.asarray([rng.below(n) for _ in range(count)], np.uint32)


class SplitMix64:
    """SplitMix64 with the reference's Rng seeding (include/common.h:44-56)."""

    M = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = (seed * 0x9E3779B97F4A7C15 + 0x1234567) & self.M

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & self.M
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
        return z ^ (z >> 31)

    def uniform(self, a: float = 0.0, b: float = 1.0) -> float:
        return a + (b - a) * ((self.next() >> 11) * (1.0 / 9007199254740992.0))

    def below(self, n: int) -> int:
        return self.next() % n
