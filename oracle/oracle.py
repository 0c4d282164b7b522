"""ORACLE - test infrastructure only.

ctypes wrapper of the C oracle (oracle/pfg_oracle.c -> oracle/_build/liboracle.so)
and, when it has been built, of the reference's own CPU code
(oracle/_ref/libpfref.so, see oracle/Makefile). Only tests/, the smoke test
and the CPU legs of bench.py import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libpfref.so"
REF_APP = HERE / "_ref" / "pathfinder_b200"
INF = 0xFFFFFFFF

u32, u64, i32, f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_double
P = C.POINTER

_lib = None
_ref = None


def _p(a, t):
    return None if a is None else a.ctypes.data_as(P(t))


def build(reference: Optional[str] = None) -> None:
    """Compiles the C oracle (and the reference shim when its sources are present)."""
    targets = ["all"]
    if reference is not None and Path(reference, "src", "cpu_sssp.cpp").exists():
        targets.append(f"REF={reference}")
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.orc_heuristic.restype = u32
        L.orc_heuristic.argtypes = [f64, f64, f64, f64, f64]
        L.orc_build_csr.restype = i32
        L.orc_build_csr.argtypes = [u32, u64, P(u32), P(u32), P(u32), P(f64), P(f64), P(u32), P(u32),
                                    P(u32), P(f64)]
        L.orc_gen_grid_road.restype = u64
        L.orc_gen_grid_road.argtypes = [u32, u32, u64, P(u32), P(u32), P(u32), P(f64), P(f64)]
        L.orc_gen_rmat_ref.restype = u64
        L.orc_gen_rmat_ref.argtypes = [u32, u32, u32, u64, P(u32), P(u32), P(u32)]
        L.orc_dijkstra.restype = f64
        L.orc_dijkstra.argtypes = [u32, P(u32), P(u32), P(u32), u32, P(u32), P(u32), P(u64)]
        L.orc_min_parent.restype = None
        L.orc_min_parent.argtypes = [u32, P(u32), P(u32), P(u32), P(u32), u32, P(u32)]
        L.orc_astar.restype = u32
        L.orc_astar.argtypes = [u32, P(u32), P(u32), P(u32), P(f64), P(f64), f64, u32, u32, i32,
                                P(u32), P(u32), P(u64)]
        L.orc_multi_source.restype = f64
        L.orc_multi_source.argtypes = [u32, P(u32), P(u32), P(u32), P(u32), u32, i32, P(u32), P(u64)]
        L.orc_max_threads.restype = i32
        L.orc_validate_path.restype = i32
        L.orc_validate_path.argtypes = [u32, P(u32), P(u32), P(u32), P(u32), u32, u32, u32, u32]
        L.orc_verify_sssp.restype = u64
        L.orc_verify_sssp.argtypes = [u32, P(u32), P(u32), P(u32), u32, P(u32), P(u32), P(u32), u32,
                                      u64, P(u64)]
        L.orc_reconstruct_path.restype = u32
        L.orc_reconstruct_path.argtypes = [P(u32), u32, u32, u32, P(u32), u32]
        L.orc_rng_stream.restype = u64
        L.orc_rng_stream.argtypes = [u64, u64, P(u64)]
        _lib = L
    return _lib


def _csr(g):
    return (np.ascontiguousarray(g.row_offsets, np.uint32), np.ascontiguousarray(g.col_indices, np.uint32),
            np.ascontiguousarray(g.weights, np.uint32))


def rng_stream(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, np.uint64)
    lib().orc_rng_stream(seed, count, _p(out, u64))
    return out


def heuristic(xv, yv, xt, yt, scale) -> int:
    return int(lib().orc_heuristic(xv, yv, xt, yt, scale))


def build_csr(n, src, dst, w, x=None, y=None):
    """Returns (row, col, w, stats dict) exactly as the reference's buildCSR would."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = np.ascontiguousarray(w, np.uint32)
    m_in = len(src)
    row = np.empty(n + 1, np.uint32)
    col = np.empty(max(1, m_in), np.uint32)
    wt = np.empty(max(1, m_in), np.uint32)
    st = np.empty(7, np.float64)
    xx = None if x is None else np.ascontiguousarray(x, np.float64)
    yy = None if y is None else np.ascontiguousarray(y, np.float64)
    rc = lib().orc_build_csr(n, m_in, _p(src, u32), _p(dst, u32), _p(w, u32), _p(xx, f64), _p(yy, f64),
                             _p(row, u32), _p(col, u32), _p(wt, u32), _p(st, f64))
    if rc != 0:
        raise RuntimeError("graph too large")
    m = int(st[0])
    stats = dict(m=m, minW=int(st[1]), maxW=int(st[2]), maxDeg=int(st[3]), avgW=float(st[4]),
                 avgDeg=float(st[5]), hScale=float(st[6]))
    return row, col[:m].copy(), wt[:m].copy(), stats


def gen_grid_road(rows, cols, seed):
    n = rows * cols
    cap = 8 * n + 8
    s, d, w = (np.empty(cap, np.uint32) for _ in range(3))
    x, y = np.empty(n, np.float64), np.empty(n, np.float64)
    m = lib().orc_gen_grid_road(rows, cols, seed, _p(s, u32), _p(d, u32), _p(w, u32), _p(x, f64), _p(y, f64))
    return n, s[:m].copy(), d[:m].copy(), w[:m].copy(), x, y


class ArcGraph:
    """A plain CSR (row_offsets, col_indices, weights, x, y, hScale) for the oracle's callers."""

    def __init__(self, row, col, w, x, y, stats):
        self.row_offsets, self.col_indices, self.weights = row, col, w
        self.x, self.y = x, y
        self.n, self.m = len(row) - 1, len(col)
        self.hScale = stats["hScale"]
        self.stats = stats


def config_grid_arcs(rows, cols, seed):
    """Arc list of the benchmark grid: vertex (r, c) at coordinates (x = c, y = r), arcs
    both ways to the right and lower neighbours, each direction with its own weight
    llround(100 * U[1, 1.5)) drawn from the reference's SplitMix64 stream in
    row-major vertex order (right pair first, then the lower pair)."""
    r, c = np.divmod(np.arange(rows * cols, dtype=np.int64), cols)
    ids = r * cols + c
    right, down = c + 1 < cols, r + 1 < rows
    cnt = 2 * right.astype(np.int64) + 2 * down.astype(np.int64)
    m = int(cnt.sum())
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    src = np.empty(m, np.int64)
    dst = np.empty(m, np.int64)
    i = start[right]
    src[i], dst[i] = ids[right], ids[right] + 1
    src[i + 1], dst[i + 1] = ids[right] + 1, ids[right]
    j = start[down] + 2 * right[down]
    src[j], dst[j] = ids[down], ids[down] + cols
    src[j + 1], dst[j + 1] = ids[down] + cols, ids[down]
    z = rng_stream(seed, m)
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    w = np.floor(100.0 * (1.0 + 0.5 * u) + 0.5)  # llround of a positive value
    x, y = c.astype(np.float64), r.astype(np.float64)
    return rows * cols, src.astype(np.uint32), dst.astype(np.uint32), w.astype(np.uint32), x, y


def config_grid(rows, cols, seed) -> ArcGraph:
    """The benchmark grid built by the oracle's buildCSR restatement."""
    n, s, d, w, x, y = config_grid_arcs(rows, cols, seed)
    row, col, wt, stats = build_csr(n, s, d, w, x, y)
    return ArcGraph(row, col, wt, x, y, stats)


def uniform_vertices(n, count, seed) -> np.ndarray:
    """`count` vertices uniform in [0, n): successive SplitMix64 outputs modulo n."""
    return (rng_stream(seed, count) % np.uint64(n)).astype(np.uint32)


def gen_rmat_ref(scale, ef, maxw, seed):
    n = 1 << scale
    cap = 2 * n * ef + 8
    s, d, w = (np.empty(cap, np.uint32) for _ in range(3))
    m = lib().orc_gen_rmat_ref(scale, ef, maxw, seed, _p(s, u32), _p(d, u32), _p(w, u32))
    return n, s[:m].copy(), d[:m].copy(), w[:m].copy()


def dijkstra(g, src):
    """Reference cpuDijkstra: (dist, parent, edges, ms)."""
    row, col, w = _csr(g)
    n = len(row) - 1
    dist = np.empty(n, np.uint32)
    par = np.empty(n, np.uint32)
    cnt = np.zeros(2, np.uint64)
    ms = lib().orc_dijkstra(n, _p(row, u32), _p(col, u32), _p(w, u32), int(src), _p(dist, u32),
                            _p(par, u32), _p(cnt, u64))
    return dist, par, int(cnt[0]), ms


def min_parent(g, dist, src):
    row, col, w = _csr(g)
    n = len(row) - 1
    dist = np.ascontiguousarray(dist, np.uint32)
    par = np.empty(n, np.uint32)
    lib().orc_min_parent(n, _p(row, u32), _p(col, u32), _p(w, u32), _p(dist, u32), int(src), _p(par, u32))
    return par


def sssp_canonical(g, src):
    """(dist, canonical smallest-index tight parent) for one source."""
    dist, _, _, _ = dijkstra(g, src)
    return dist, min_parent(g, dist, src)


def astar(g, src, dst, use_heuristic=True):
    """Reference cpuAStar: (dist, path list, edges, ms)."""
    row, col, w = _csr(g)
    n = len(row) - 1
    x = None if g.x is None else np.ascontiguousarray(g.x, np.float64)
    y = None if g.y is None else np.ascontiguousarray(g.y, np.float64)
    path = np.empty(n + 1, np.uint32)
    ln = C.c_uint32(0)
    cnt = np.zeros(3, np.uint64)
    d = lib().orc_astar(n, _p(row, u32), _p(col, u32), _p(w, u32), _p(x, f64), _p(y, f64),
                        float(g.hScale), int(src), int(dst), 1 if use_heuristic else 0, _p(path, u32),
                        C.byref(ln), _p(cnt, u64))
    return int(d), path[: ln.value].tolist(), int(cnt[0]), cnt[2] / 1e6


def multi_source(g, srcs, threads=0, keep=False):
    """Reference cpuMultiSource (OpenMP over sources): (ms, dist [k, n] or None, edges)."""
    row, col, w = _csr(g)
    n = len(row) - 1
    srcs = np.ascontiguousarray(srcs, np.uint32)
    out = np.empty(len(srcs) * n, np.uint32) if keep else None
    edges = C.c_uint64(0)
    ms = lib().orc_multi_source(n, _p(row, u32), _p(col, u32), _p(w, u32), _p(srcs, u32), len(srcs),
                                int(threads), _p(out, u32), C.byref(edges))
    return ms, (None if out is None else out.reshape(len(srcs), n)), int(edges.value)


def max_threads() -> int:
    return int(lib().orc_max_threads())


def validate_path(g, path, src, dst, expected) -> bool:
    row, col, w = _csr(g)
    p = np.ascontiguousarray(path, np.uint32) if len(path) else np.zeros(1, np.uint32)
    return bool(lib().orc_validate_path(len(row) - 1, _p(row, u32), _p(col, u32), _p(w, u32), _p(p, u32),
                                        len(path), int(src), int(dst), int(expected)))


def verify_sssp(g, src, ref_dist, dist, parent, samples=64, seed=0):
    """The reference's three verifySSSP checks; returns the report dict."""
    row, col, w = _csr(g)
    rep = np.zeros(6, np.uint64)
    rd = np.ascontiguousarray(ref_dist, np.uint32)
    d = np.ascontiguousarray(dist, np.uint32)
    p = np.ascontiguousarray(parent, np.uint32)
    lib().orc_verify_sssp(len(row) - 1, _p(row, u32), _p(col, u32), _p(w, u32), int(src), _p(rd, u32),
                          _p(d, u32), _p(p, u32), int(samples), int(seed), _p(rep, u64))
    keys = ["distChecked", "distMismatch", "treeChecked", "treeErrors", "pathsChecked", "pathErrors"]
    r = {k: int(v) for k, v in zip(keys, rep)}
    r["errors"] = r["distMismatch"] + r["treeErrors"] + r["pathErrors"]
    return r


# ---------------------------------------------------------------------------
# The reference's own CPU code (oracle/_ref/libpfref.so), when built.
# ---------------------------------------------------------------------------
def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
        R = C.CDLL(str(REF_LIB))
        R.ref_gen_grid_road.restype = C.c_void_p
        R.ref_gen_grid_road.argtypes = [u32, u32, u64]
        R.ref_gen_rmat.restype = C.c_void_p
        R.ref_gen_rmat.argtypes = [u32, u32, u32, u64]
        R.ref_build_csr.restype = C.c_void_p
        R.ref_build_csr.argtypes = [u32, u64, P(u32), P(u32), P(u32), P(f64), P(f64)]
        R.ref_wrap_csr.restype = C.c_void_p
        R.ref_wrap_csr.argtypes = [u32, u32, P(u32), P(u32), P(u32), P(f64), P(f64), f64]
        R.ref_free.argtypes = [C.c_void_p]
        for nm in ("ref_n", "ref_m"):
            getattr(R, nm).restype = u32
            getattr(R, nm).argtypes = [C.c_void_p]
        for nm in ("ref_row", "ref_col", "ref_w"):
            getattr(R, nm).restype = P(u32)
            getattr(R, nm).argtypes = [C.c_void_p]
        for nm in ("ref_x", "ref_y"):
            getattr(R, nm).restype = P(f64)
            getattr(R, nm).argtypes = [C.c_void_p]
        R.ref_stats.argtypes = [C.c_void_p, P(f64)]
        R.ref_dijkstra.restype = f64
        R.ref_dijkstra.argtypes = [C.c_void_p, u32, P(u32), P(u32), P(u64)]
        R.ref_astar.restype = u32
        R.ref_astar.argtypes = [C.c_void_p, u32, u32, i32, P(u32), P(u32), P(f64), P(u64)]
        R.ref_multi_source.restype = f64
        R.ref_multi_source.argtypes = [C.c_void_p, P(u32), u32, i32, P(u32), P(u64)]
        R.ref_max_threads.restype = i32
        R.ref_verify_sssp.restype = u64
        R.ref_verify_sssp.argtypes = [C.c_void_p, u32, P(u32), P(u32), P(u32), u32, u64, P(u64)]
        R.ref_validate_path.restype = i32
        R.ref_validate_path.argtypes = [C.c_void_p, P(u32), u32, u32, u32, u32]
        R.ref_pick_sources.argtypes = [C.c_void_p, u32, u64, P(u32)]
        R.ref_heuristic.restype = u32
        R.ref_heuristic.argtypes = [f64, f64, f64, f64, f64]
        R.ref_load_dimacs.restype = C.c_void_p
        R.ref_load_dimacs.argtypes = [C.c_char_p, C.c_char_p]
        R.ref_load_snap.restype = C.c_void_p
        R.ref_load_snap.argtypes = [C.c_char_p, i32, u32, u64]
        R.ref_load_binary.restype = C.c_void_p
        R.ref_load_binary.argtypes = [C.c_char_p]
        R.ref_save_binary.restype = i32
        R.ref_save_binary.argtypes = [C.c_void_p, C.c_char_p]
        _ref = R
    return _ref


class RefGraph:
    """A CSRGraph object living inside the reference's own code."""

    def __init__(self, handle):
        self.h = handle

    @staticmethod
    def wrap(g) -> "RefGraph":
        row, col, w = _csr(g)
        x = None if g.x is None else np.ascontiguousarray(g.x, np.float64)
        y = None if g.y is None else np.ascontiguousarray(g.y, np.float64)
        return RefGraph(ref().ref_wrap_csr(len(row) - 1, len(col), _p(row, u32), _p(col, u32), _p(w, u32),
                                           _p(x, f64), _p(y, f64), float(g.hScale)))

    def __del__(self):
        try:
            if self.h:
                ref().ref_free(self.h)
        except Exception:
            pass

    def arrays(self):
        R = ref()
        n, m = R.ref_n(self.h), R.ref_m(self.h)
        row = np.ctypeslib.as_array(R.ref_row(self.h), shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(R.ref_col(self.h), shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        w = np.ctypeslib.as_array(R.ref_w(self.h), shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        xp, yp = R.ref_x(self.h), R.ref_y(self.h)
        x = np.ctypeslib.as_array(xp, shape=(n,)).copy() if xp else None
        y = np.ctypeslib.as_array(yp, shape=(n,)).copy() if yp else None
        st = np.empty(7, np.float64)
        R.ref_stats(self.h, _p(st, f64))
        stats = dict(m=int(st[0]), minW=int(st[1]), maxW=int(st[2]), maxDeg=int(st[3]), avgW=float(st[4]),
                     avgDeg=float(st[5]), hScale=float(st[6]))
        return row, col, w, x, y, stats

    def dijkstra(self, src):
        n = ref().ref_n(self.h)
        d, p = np.empty(n, np.uint32), np.empty(n, np.uint32)
        e = C.c_uint64(0)
        ms = ref().ref_dijkstra(self.h, int(src), _p(d, u32), _p(p, u32), C.byref(e))
        return d, p, int(e.value), ms

    def astar(self, src, dst, use_h=True):
        n = ref().ref_n(self.h)
        path = np.empty(n + 1, np.uint32)
        ln = C.c_uint32(0)
        ms = C.c_double(0)
        e = C.c_uint64(0)
        d = ref().ref_astar(self.h, int(src), int(dst), 1 if use_h else 0, _p(path, u32), C.byref(ln),
                            C.byref(ms), C.byref(e))
        return int(d), path[: ln.value].tolist(), int(e.value), ms.value

    def multi_source(self, srcs, threads=0, keep=False):
        n = ref().ref_n(self.h)
        srcs = np.ascontiguousarray(srcs, np.uint32)
        out = np.empty(len(srcs) * n, np.uint32) if keep else None
        e = C.c_uint64(0)
        ms = ref().ref_multi_source(self.h, _p(srcs, u32), len(srcs), int(threads), _p(out, u32), C.byref(e))
        return ms, (None if out is None else out.reshape(len(srcs), n)), int(e.value)

    def pick_sources(self, count, seed):
        out = np.empty(count, np.uint32)
        ref().ref_pick_sources(self.h, count, seed, _p(out, u32))
        return out

    def save_binary(self, path) -> bool:
        """The reference's saveBinary (PFCSR001 cache file)."""
        return ref().ref_save_binary(self.h, str(path).encode()) == 1


def _loaded(h) -> Optional[RefGraph]:
    return RefGraph(h) if h else None


def ref_load_dimacs(gr, co=None) -> Optional[RefGraph]:
    """The reference's loadDIMACS + buildCSR; None when its loader fails."""
    return _loaded(ref().ref_load_dimacs(str(gr).encode(), None if co is None else str(co).encode()))


def ref_load_snap(path, symmetrize=True, max_w=1000, seed=2026) -> Optional[RefGraph]:
    """The reference's loadSNAP + buildCSR; None when its loader fails."""
    return _loaded(ref().ref_load_snap(str(path).encode(), 1 if symmetrize else 0, max_w, seed))


def ref_load_binary(path) -> Optional[RefGraph]:
    """The reference's loadBinary (PFCSR001); None when its loader fails."""
    return _loaded(ref().ref_load_binary(str(path).encode()))


def ref_gen_grid_road(rows, cols, seed) -> RefGraph:
    return RefGraph(ref().ref_gen_grid_road(rows, cols, seed))


def ref_gen_rmat(scale, ef, maxw, seed) -> RefGraph:
    return RefGraph(ref().ref_gen_rmat(scale, ef, maxw, seed))


def ref_build_csr(n, src, dst, w, x=None, y=None) -> RefGraph:
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = np.ascontiguousarray(w, np.uint32)
    xx = None if x is None else np.ascontiguousarray(x, np.float64)
    yy = None if y is None else np.ascontiguousarray(y, np.float64)
    return RefGraph(ref().ref_build_csr(n, len(src), _p(src, u32), _p(dst, u32), _p(w, u32), _p(xx, f64),
                                        _p(yy, f64)))
