"""Serving A* queries with continuous batching (C ABI: pfg_server_*).

    srv = GpuServer(g, slots=64)     # slots=0: as many as 60 % of the free device memory holds
    qid = srv.submit(s, t)          # queued on the host
    srv.step(max_rounds=32)         # admit into free slots, run <= 32 device rounds, retire finished
    for r in srv.results(): ...     # id, src, dst, dist, slot, submit_us, admit_us, finish_us

run_poisson() replays a Poisson arrival stream against a server in real time and
reports p50 / p99 latency (from each query's scheduled arrival to the step that
returned its result) and the achieved queries per second.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .graphs import CSRGraph
from .solver import GpuOptions


from ._native import PfgQueryResult


def _lib():
    return N.load()


class GpuServer:
    def __init__(self, g: CSRGraph, slots: int = 64, opt: Optional[GpuOptions] = None, device: int = 0):
        self._lib = _lib()
        self.g = g
        self._row = np.ascontiguousarray(g.row_offsets, np.uint32)
        self._col = np.ascontiguousarray(g.col_indices, np.uint32)
        self._w = np.ascontiguousarray(g.weights, np.uint32)
        x = None if g.x is None else np.ascontiguousarray(g.x, np.float64)
        y = None if g.y is None else np.ascontiguousarray(g.y, np.float64)
        c = (opt or GpuOptions()).to_c()
        h = C.c_void_p()
        N.check(self._lib.pfg_server_create(N.ptr(self._row, N.u32), N.ptr(self._col, N.u32),
                                            N.ptr(self._w, N.u32), N.ptr(x, N.f64), N.ptr(y, N.f64), g.n, g.m,
                                            float(g.hScale), float(g.avgW), float(g.avgDeg), int(slots),
                                            C.byref(c), int(device), C.byref(h)))
        self._h = h
        self.slots = int(self._lib.pfg_server_slots(h))  # chosen by device memory when slots = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pfg_server_destroy(self._h)
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

    def submit(self, src: int, dst: int) -> int:
        qid = N.u64()
        N.check(self._lib.pfg_server_submit(self._h, int(src), int(dst), C.byref(qid)))
        return int(qid.value)

    def step(self, max_rounds: int = 32) -> Tuple[int, int]:
        a, d = N.u32(), N.u32()
        N.check(self._lib.pfg_server_step(self._h, int(max_rounds), C.byref(a), C.byref(d)))
        return int(a.value), int(d.value)

    def results(self) -> List[Dict]:
        out = []
        buf = (PfgQueryResult * 256)()
        while True:
            k = N.u32()
            N.check(self._lib.pfg_server_results(self._h, buf, 256, C.byref(k)))
            for i in range(k.value):
                r = buf[i]
                out.append(dict(id=r.id, src=r.src, dst=r.dst, dist=r.dist, slot=r.slot, submit_us=r.submit_us,
                                admit_us=r.admit_us, finish_us=r.finish_us))
            if k.value < 256:
                return out

    def pending(self) -> int:
        return int(self._lib.pfg_server_pending(self._h))

    def in_flight(self) -> int:
        return int(self._lib.pfg_server_in_flight(self._h))

    def now_us(self) -> float:
        return float(self._lib.pfg_server_now_us(self._h))

    def set_policy(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        s = self._lib.pfg_server_solver(self._h)
        N.check(self._lib.pfg_set_policy(C.c_void_p(s), N.ptr(p, N.f32), p.size))

    def drain(self, max_rounds: int = 32, max_steps: int = 1_000_000) -> List[Dict]:
        """Steps until every submitted query has finished; returns their results."""
        out = []
        for _ in range(max_steps):
            if self.pending() == 0 and self.in_flight() == 0:
                break
            self.step(max_rounds)
            out += self.results()
        return out + self.results()


def answer_all(server: GpuServer, pairs: Sequence[Tuple[int, int]], max_rounds: int = 8) -> List[int]:
    """Target distances of `pairs` (in order), all admitted at once and drained."""
    ids = [server.submit(int(s), int(t)) for s, t in pairs]
    got = {r["id"]: r["dist"] for r in server.drain(max_rounds=max_rounds)}
    return [got[q] for q in ids]


def run_poisson(server: GpuServer, pairs: Sequence[Tuple[int, int]], rate_qps: float, max_rounds: int = 32,
                seed: int = 0, time_limit_s: float = 120.0) -> Dict:
    """Real-time replay of Poisson arrivals at `rate_qps`; latency = finish - scheduled arrival."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1e6 / rate_qps, size=len(pairs))
    arrive = np.cumsum(gaps) - gaps[0]
    t0 = server.now_us()
    sched = {}
    nxt = 0
    done = []
    steps = 0
    while len(done) < len(pairs):
        now = server.now_us() - t0
        if now > time_limit_s * 1e6:
            break
        while nxt < len(pairs) and arrive[nxt] <= now:
            qid = server.submit(*pairs[nxt])
            sched[qid] = t0 + arrive[nxt]
            nxt += 1
        if server.pending() == 0 and server.in_flight() == 0:
            if nxt < len(pairs):
                while server.now_us() - t0 < arrive[nxt]:
                    pass
            continue
        server.step(max_rounds)
        steps += 1
        done += server.results()
    lat = np.array([(r["finish_us"] - sched[r["id"]]) / 1e3 for r in done])
    span_s = (max(r["finish_us"] for r in done) - t0) / 1e6 if done else float("nan")
    return {"offered_qps": rate_qps, "queries": len(done), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "achieved_qps": len(done) / span_s, "steps": steps, "results": done}
