"""Benchmark of the SSSP hot path: batched Delta-stepping on the 1000 x 1000 grid road graph.

One step = one multi-source SSSP launch (reference GpuSolver::multiSource,
src/gpu_sssp.cu:553-569): K sources on the 1000x1000 grid (n = 10^6,
m = 3,996,000 arcs, w = llround(100 * U[1, 1.5)), seed 2026) relaxed by one
persistent kernel, fixed automatic Delta, buckets drained asynchronously (the
engine's default schedule). Metric: GTEPS = reachable arcs of all K instances /
step time (the reference's TEPS definition, src/main.cpp:209-213, aggregated
over the batch).

  value  device time of the step with the graph, sources and working set resident
         in HBM (CUDA events on the solver's stream, L2 flushed between steps); the
         launch shape (threads per CTA x CTAs per SM) is the fastest of the
         autotuner's candidates on this workload, timed before the warm-up
  e2e    the same steps through the C ABI as a stream of the reference's multiSource
         calls with distOut (pfg_run_dist_async, then pfg_dist_wait): per step the H2D of
         the K sources from pinned memory, the run, and the K*n distances split from the
         packed words on the device and copied into pinned memory, the copy of one step
         overlapping the next step's kernel; timed on the device from before the first
         step to after the last copy. e2e.sync_value is the one-call-at-a-time form
         (pfg_run + pfg_copy_dist)
  --impl reference   the reference's own cpuMultiSource (OpenMP, every host thread)
         on the same graph and sources, compiled from its sources into oracle/_ref
  extras (N = 1, skipped with --no-extras): single-source Delta / Frontier / Naive and
         256 A* pairs on the same grid; R-MAT-20 learned policy vs fixed Delta;
         the uneven batch (64 sources on a 1024x1024 grid + 256 grids of 32..316 per
         side) in one launch replayed from a CUDA graph; A* serving on the
         2048x2048 road-like graph under Poisson arrivals (p50 / p99 latency).

Multi-GPU: replicas (each rank runs its own batch of sources; no collective on the
data path), value = all ranks' arcs / max step time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID_SIDE = 1000
SEED = 2026
BATCH = 64


def HEADLINE_OPTIONS():
    """Fixed automatic Delta, default schedule (asynchronous buckets), blind atomicMin."""
    from pathfinding_gpu_b200 import GpuOptions, AtomicMode
    return GpuOptions(atomic=AtomicMode.MinNoCheck)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--no-extras", action="store_true", help="skip the single-source / A* extras")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU, torchrun env)
# ---------------------------------------------------------------------------
def Dist(n_gpus: int):
    """Replica process group (NCCL), one process per GPU; see pathfinding_gpu_b200/replicas.py."""
    from pathfinding_gpu_b200.replicas import ReplicaGroup
    return ReplicaGroup(backend="nccl" if int(os.environ.get("WORLD_SIZE", "1")) > 1 else None)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []  # (host time of arrival, csv line)
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def start_window(self):
        self.window = [time.perf_counter(), None]

    def end_window(self):
        if self.window:
            self.window[1] = time.perf_counter()

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if self.window and self.window[1] is not None:
            # samples that arrived while the timed region ran (lines come a few ms late)
            inside = [x for x in lines if self.window[0] <= x[0] <= self.window[1] + 0.03]
            lines = inside or lines[-1:]
        for _, ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_key: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(kernel_key)
    except Exception:
        return None


def workload(rank: int, batch: int):
    import pathfinding_gpu_b200 as pf
    g = pf.grid(GRID_SIDE, GRID_SIDE, SEED)
    srcs = pf.uniform_vertices(g.n, batch, SEED + 1000 * rank)
    return g, srcs


def reachable_stats(g, dist_rows):
    """Reachable arcs and vertices summed over instances."""
    deg = np.diff(g.row_offsets).astype(np.int64)
    mr = nr = 0
    for d in dist_rows:
        r = d != 0xFFFFFFFF
        nr += int(r.sum())
        mr += int(deg[r].sum())
    return mr, nr


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def run_ours(args, D):
    import torch
    import pathfinding_gpu_b200 as pf
    from pathfinding_gpu_b200 import GpuOptions

    torch.cuda.set_device(D.local)
    g, srcs = workload(D.rank, args.batch)
    K = args.batch
    solver = pf.GpuSolver(g, K, device=D.local)
    stream = torch.cuda.ExternalStream(solver.stream(), device=D.local)
    opt = HEADLINE_OPTIONS()
    lib = solver._lib
    import ctypes as C
    from pathfinding_gpu_b200 import _native as N

    d_srcs = torch.from_numpy(srcs.astype(np.int32)).to(f"cuda:{D.local}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{D.local}")

    # Launch shape: the autotuner's launch-shape candidates timed on this
    # workload before the warm-up (median of 3 runs each, L2 flushed); Delta
    # stays the automatic value and the schedule the default.
    from dataclasses import replace
    from pathfinding_gpu_b200.autotune import LAUNCH_SHAPES
    shape_ms = {}
    for bsz, bps in LAUNCH_SHAPES:
        trial = replace(opt, blockSize=bsz, blocksPerSM=bps)
        ts = []
        for _ in range(3):
            flush.zero_()
            torch.cuda.synchronize()
            ts.append(solver.run_state(srcs, trial, copy=False)[1])
        shape_ms[f"{bsz}x{bps}"] = round(statistics.median(ts), 3)
    bsz, bps = min(LAUNCH_SHAPES, key=lambda s: shape_ms[f"{s[0]}x{s[1]}"])
    opt = replace(opt, blockSize=bsz, blocksPerSM=bps)
    copt = opt.to_c()

    def device_step():
        N.check(lib.pfg_run_async(solver.handle, C.c_void_p(d_srcs.data_ptr()), K, 0, 0, C.byref(copt)))

    def finish():
        st = N.PfgStats()
        N.check(lib.pfg_finish(solver.handle, C.byref(st)))
        return st

    # reachable arcs from one full run (also a parity spot check against the oracle on rank 0)
    stats0, _, state = solver.run_state(srcs, opt)
    dist, _ = pf.unpack(state)
    dist = dist.reshape(K, g.n)
    m_r, n_r = reachable_stats(g, dist)

    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.zero_()
        device_step()
        finish()
    D.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    launches = 0
    with ClockSampler(D.local) as clk:
        clk.start_window()
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # L2 flush between timed steps (256 MB > 126 MB L2)
                evs[i][0].record(stream)
            device_step()
            launches += 1
            evs[i][1].record(stream)
            finish()
        torch.cuda.synchronize()
        clk.end_window()
    D.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    local_total = sum(step_ms)
    total_ms = D.max(local_total)
    ms_per_step = total_ms / args.steps
    arcs_all = D.sum(float(m_r))
    value = arcs_all / (ms_per_step * 1e-3) / 1e9

    # ---- roofline of the persistent kernel (one launch per step) ----
    bytes_alg = 16.0 * m_r + 20.0 * n_r
    achieved = bytes_alg / (statistics.mean(step_ms) * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic("k_persistent_grid1000_k64")

    # ---- end to end through the C ABI with host buffers ----
    # Streamed multiSource (pfg_run_dist_async / pfg_dist_wait): every step copies
    # its K sources from pinned memory and its K*n distances back into pinned
    # memory; the copy of one step's distances overlaps the next step's kernel.
    h_dist = [torch.empty(K * g.n, dtype=torch.int32).pin_memory() for _ in range(2)]
    h_srcs = np.ascontiguousarray(srcs, np.uint32)
    st = N.PfgStats()
    as_u32 = lambda tsr: C.cast(C.c_void_p(tsr.data_ptr()), C.POINTER(C.c_uint32))

    def streamed(i):
        N.check(lib.pfg_run_dist_async(solver.handle, N.ptr(h_srcs, N.u32), K, C.byref(copt),
                                       as_u32(h_dist[i % 2]), C.byref(st)))

    for i in range(args.warmup):
        streamed(i)
    N.check(lib.pfg_dist_wait(solver.handle, C.byref(st)))
    for h in h_dist:
        h.fill_(-1)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for i in range(args.steps):
        streamed(i)
    N.check(lib.pfg_dist_wait(solver.handle, C.byref(st)))
    b.record(stream)
    torch.cuda.synchronize()
    e2e_ms = D.max(a.elapsed_time(b) / args.steps)
    e2e_value = arcs_all / (e2e_ms * 1e-3) / 1e9
    # every copied-back result must be the device result
    for h in h_dist[:min(2, args.steps)]:
        got = h.numpy().view(np.uint32).reshape(K, g.n)
        assert np.array_equal(got, dist), "e2e result differs from the device-resident run"
    # the synchronous form (one multiSource call at a time: run, then copy), for reference
    ms_c = C.c_float()
    sync_ms = []
    for i in range(3):
        a2, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a2.record(stream)
        N.check(lib.pfg_run(solver.handle, N.ptr(h_srcs, N.u32), K, 0, 0, C.byref(copt), C.byref(st),
                            None, C.byref(ms_c)))
        N.check(lib.pfg_copy_dist(solver.handle, 0, K * g.n, as_u32(h_dist[0])))
        b2.record(stream)
        torch.cuda.synchronize()
        sync_ms.append(a2.elapsed_time(b2))
    e2e_sync_ms = D.max(statistics.median(sync_ms))

    result = {
        "metric": "GTEPS (reachable arcs / s, SSSP Delta-stepping, batch of sources)",
        "value": round(value, 4), "unit": "GTEPS", "n_gpus": D.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"grid{GRID_SIDE}x{GRID_SIDE} multiSource K={K} Delta-stepping",
                   "graph": f"grid {GRID_SIDE}x{GRID_SIDE}, 4-neighbour arcs both ways, "
                            f"w=llround(100*U[1,1.5)), seed {SEED}",
                   "n": g.n, "m": g.m, "batch": K, "delta": stats0.delta, "algo": "DeltaStep",
                   "schedule": opt.schedule.name, "mapping": opt.mapping.name, "atomic": opt.atomic.name,
                   "block": opt.blockSize, "ctas_per_sm": opt.blocksPerSM,
                   "launch_shape_ms": shape_ms, "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"replicas x{D.world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 5), "traffic": traffic,
                     "peak_kind": peak_kind,
                     "bytes_alg_per_launch": bytes_alg,
                     "bytes_model": "16 B per reachable arc + 20 B per reachable vertex, per instance"},
        "e2e": {"value": round(e2e_value, 4), "unit": "GTEPS", "h2d_bytes_per_step": 4 * K + 256,
                "d2h_bytes_per_step": 4 * K * g.n + 256, "ms_per_step": round(e2e_ms, 4),
                "api": "pfg_run_dist_async / pfg_dist_wait (C ABI; streamed multiSource with distOut: "
                       "each step's distance copy overlaps the next step's kernel) with pinned host buffers",
                "sync_value": round(arcs_all / (e2e_sync_ms * 1e-3) / 1e9, 4),
                "sync_ms_per_step": round(e2e_sync_ms, 4),
                "sync_api": "pfg_run + pfg_copy_dist, one call completed before the next"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "stats": {"rounds": stats0.rounds, "buckets": stats0.buckets,
                  "edges_scanned": stats0.edgesScanned, "work_per_m": stats0.edgesScanned / max(1, m_r),
                  "atomics": stats0.atomicsIssued},
    }
    solver.close()
    return result, g, srcs


def cpu_baseline(g, srcs, sample: int):
    """The reference's cpuMultiSource (every host thread) on a bounded sample."""
    from oracle import oracle as O
    srcs = np.asarray(srcs[:sample], np.uint32)
    if O.ref_available():
        R = O.RefGraph.wrap(g)
        ms, _, edges = R.multi_source(srcs, 0, False)
        threads = O.ref().ref_max_threads()
        kind = "reference"
    else:
        ms, _, edges = O.multi_source(g, srcs, 0, False)
        threads = O.max_threads()
        kind = "port"
    deg = np.diff(g.row_offsets).astype(np.int64)
    # grid graphs are strongly connected: every arc is reachable from every source
    m_r = int(deg.sum()) * len(srcs)
    return {"value": round(m_r / (ms * 1e-3) / 1e9, 4), "unit": "GTEPS", "cores": int(threads),
            "kind": kind, "ms": round(ms, 2),
            "sample": f"{len(srcs)} of the step's sources, cpuMultiSource OpenMP x{threads}"}


def _opt_dict(o):
    from dataclasses import asdict
    return {k: (v.name if hasattr(v, "name") else v) for k, v in asdict(o).items()}


def cpu_single_thread(g, gr, src, pairs):
    """cpuDijkstra (1 thread) on the 1000x1000 grid and R-MAT-20 and cpuAStar on a sample of
    the grid's 256 pairs, from the reference's own code (oracle/_ref) when built, else the
    oracle's restatement."""
    from oracle import oracle as O
    use_ref = O.ref_available()
    out = {"cores": 1, "kind": "reference" if use_ref else "port"}
    for name, graph, srcs in (("grid1000", g, [src] + pf_sources(g, 2)), ("rmat20", gr, pf_sources(gr, 3))):
        R = O.RefGraph.wrap(graph) if use_ref else None
        ms = []
        for s_ in srcs:
            ms.append(R.dijkstra(int(s_))[3] if use_ref else O.dijkstra(graph, int(s_))[3])
        deg = np.diff(graph.row_offsets).astype(np.int64)
        out[f"{name}_cpuDijkstra_ms"] = round(statistics.median(ms), 2)
        out[f"{name}_cpuDijkstra_sources"] = len(srcs)
    R = O.RefGraph.wrap(g) if use_ref else None
    ams = []
    for a, b in pairs[:64]:
        ams.append(R.astar(int(a), int(b))[3] if use_ref else O.astar(g, int(a), int(b))[3])
    out["grid1000_cpuAStar_ms"] = {"mean": round(float(np.mean(ams)), 3), "pairs": len(ams),
                                   "sample": "the first 64 of the 256 pairs"}
    return out


def pf_sources(graph, k):
    import pathfinding_gpu_b200 as pf
    return pf.pick_sources(graph, k, 99).tolist()


def _median_ms(fn, reps=5):
    fn()
    return statistics.median(fn() for _ in range(reps))


def extras(g):
    """The other workloads, timed on the device (reported beside the headline)."""
    import pathfinding_gpu_b200 as pf
    from pathfinding_gpu_b200 import GpuOptions, GpuAlgo, Policy
    out = {}
    t0 = time.perf_counter()
    # --- the 1000x1000 grid: single-source modes and 256 A* pairs ---
    pairs = pf.uniform_vertices(g.n, 2 * 256, SEED + 7).reshape(-1, 2)
    src = int(pf.uniform_vertices(g.n, 1, SEED)[0])
    with pf.GpuSolver(g, 1) as s:
        for algo in (GpuAlgo.DeltaStep, GpuAlgo.Frontier, GpuAlgo.NaiveRelax):
            o = GpuOptions(algo=algo)
            out[f"grid1000_sssp_{algo.name}_ms"] = round(_median_ms(lambda: s.run_state([src], o, copy=False)[1], 3), 3)
        ts = [s.run_state([int(a)], GpuOptions(), astar=True, dst=int(b), copy=False)[1] for a, b in pairs]
        out["grid1000_astar_256_pairs_ms"] = {"mean": round(float(np.mean(ts)), 3),
                                              "p50": round(float(np.percentile(ts, 50)), 3),
                                              "p99": round(float(np.percentile(ts, 99)), 3)}
    # --- aggregate throughput against the batch size (roofline per launch) ---
    from pathfinding_gpu_b200 import policy as P
    peak, _ = measured_peaks()
    sweep = {}
    Ks = (16, 32, 64, 128, 256)
    srcs_all = pf.uniform_vertices(g.n, max(Ks), SEED)
    from dataclasses import replace
    from pathfinding_gpu_b200 import Schedule
    with pf.GpuSolver(g, max(Ks)) as s:
        for K in Ks:
            # the drain kind and launch shape the autotuner chooses between, timed per batch size
            cands = {}
            # (Auto: a shared window below 96 sources, a window per instance from 96 on)
            for sched in (Schedule.Auto, Schedule.Warp):
                for bsz, bps in ((256, 4), (512, 2), (1024, 1)):
                    o = replace(HEADLINE_OPTIONS(), schedule=sched, blockSize=bsz, blocksPerSM=bps)
                    cands[f"{sched.name}/{bsz}x{bps}"] = round(
                        _median_ms(lambda: s.run_state(srcs_all[:K], o, copy=False)[1], 3), 3)
            best = min(cands, key=cands.get)
            ms = cands[best]
            b_alg = K * (16.0 * g.m + 20.0 * g.n)  # grid: every arc and vertex reachable
            sweep[str(K)] = {"ms": ms, "best": best, "gteps": round(K * g.m / ms / 1e6, 3),
                             "roofline_frac": round(b_alg / (ms * 1e-3) / 1e9 / peak, 4), "candidates_ms": cands}
    out["grid1000_batch_sweep"] = sweep
    # the learned policy on the step's own workload (K = 64), same engine and sources
    if P.WEIGHTS.exists():
        with pf.GpuSolver(g, 64) as s:
            s.set_policy(P.load())
            fixed = HEADLINE_OPTIONS()
            learned = replace(HEADLINE_OPTIONS(), policy=Policy.Learned)
            tf = _median_ms(lambda: s.run_state(srcs_all[:64], fixed, copy=False)[1], 3)
            tl = _median_ms(lambda: s.run_state(srcs_all[:64], learned, copy=False)[1], 3)
            a = s.run_state(srcs_all[:64], fixed)[2]
            st_l, _, b = s.run_state(srcs_all[:64], learned)
            out["grid1000_k64_learned_vs_fixed"] = {"fixed_ms": round(tf, 3), "learned_ms": round(tl, 3),
                                                    "speedup": round(tf / tl, 3), "buckets_learned": st_l.buckets,
                                                    "identical_state": bool(np.array_equal(a, b))}
    # --- R-MAT scale 20: batched multi-source throughput, learned policy vs fixed automatic Delta ---
    from pathfinding_gpu_b200 import policy as P
    gr = pf.rmat(20, 16, seed=SEED)
    deg = np.diff(gr.row_offsets).astype(np.int64)
    rsrcs = pf.pick_sources(gr, 16, SEED)
    with pf.GpuSolver(gr, 16) as s:
        o = HEADLINE_OPTIONS()
        _, _, state = s.run_state(rsrcs, o)
        dist = pf.unpack(state)[0].reshape(16, gr.n)
        reach = dist != 0xFFFFFFFF
        m_r = int((deg[None, :] * reach).sum())
        n_r = int(reach.sum())
        shapes = {}
        for sched in (Schedule.Auto, Schedule.Warp):
            for bsz, bps in ((256, 4), (1024, 1)):
                oo = replace(o, schedule=sched, blockSize=bsz, blocksPerSM=bps)
                shapes[f"{sched.name}/{bsz}x{bps}"] = round(_median_ms(lambda: s.run_state(rsrcs, oo, copy=False)[1], 3), 3)
        best = min(shapes, key=shapes.get)
        ms = shapes[best]
        out["rmat20_batch16"] = {"ms": ms, "best": best, "candidates_ms": shapes, "gteps": round(m_r / ms / 1e6, 3),
                                 "roofline_frac": round((16.0 * m_r + 20.0 * n_r) / (ms * 1e-3) / 1e9 / peak, 4),
                                 "reachable_arcs": m_r}
    if P.WEIGHTS.exists():
        with pf.GpuSolver(gr, 1) as s:
            s.set_policy(P.load())
            rows = []
            for src in pf.pick_sources(gr, 3, 99).tolist():
                fixed = GpuOptions(blockSize=1024)
                learned = GpuOptions(blockSize=1024, policy=Policy.Learned)
                tf = _median_ms(lambda: s.run_state([src], fixed, copy=False)[1])
                tl = _median_ms(lambda: s.run_state([src], learned, copy=False)[1])
                st_f, _, a = s.run_state([src], fixed)
                st_l, _, b = s.run_state([src], learned)
                rows.append({"src": src, "fixed_ms": round(tf, 3), "learned_ms": round(tl, 3),
                             "speedup": round(tf / tl, 3), "identical_state": bool(np.array_equal(a, b)),
                             "work_per_m_fixed": round(st_f.edgesScanned / gr.m, 3),
                             "work_per_m_learned": round(st_l.edgesScanned / gr.m, 3)})
            out["rmat20_learned_vs_fixed"] = {"median_speedup": statistics.median(r["speedup"] for r in rows),
                                              "runs": rows}
    # --- the reference's own CPU code, single thread, on the same inputs ---
    out["cpu_reference_single_thread"] = cpu_single_thread(g, gr, src, pairs)
    # --- uneven batch in one launch, schedule from the autotuner, replayed from a CUDA graph ---
    from pathfinding_gpu_b200.batch import GpuBatch
    from pathfinding_gpu_b200 import autotune
    import tempfile
    big = pf.grid(1024, 1024, SEED)
    small = pf.grid_batch(256, 32, 316, SEED)
    graphs = [big] + small
    inst = [(0, int(v)) for v in pf.uniform_vertices(big.n, 64, SEED)]
    inst += [(i + 1, int(pf.uniform_vertices(gs.n, 1, 100 + i)[0])) for i, gs in enumerate(small)]
    states = 64 * big.n + sum(gs.n for gs in small)
    with GpuBatch(graphs, max_states=states, max_instances=len(inst)) as b:
        b.set_instances(inst)
        o_default = GpuOptions(atomic=pf.AtomicMode.MinNoCheck)
        default_ms = _median_ms(lambda: b.run(o_default)[1], 3)
        os.environ.setdefault("PFG_TUNE_CACHE", str(Path(tempfile.gettempdir()) / "pfg_bench_tune.json"))
        key = f"batch-{len(graphs)}graphs-{len(inst)}inst-{states}states-{big.n}big"
        auto_delta = b.run(o_default)[0].delta
        tuned, tuned_ms, log = autotune.tune(lambda o: b.run(o)[1], o_default, auto_delta, reps=2,
                                             key=key, use_cache=False)
        run_ms = _median_ms(lambda: b.run(tuned)[1], 3)
        b.capture(tuned)
        rep_ms = _median_ms(lambda: b.replay()[1], 5)
        arcs = 64 * big.m + sum(gs.m for gs in small)
        out["batch_uneven"] = {"instances": len(inst), "states": states, "arcs": arcs,
                               "default_options_ms": round(default_ms, 3),
                               "tuned_key": key, "tuned_options": _opt_dict(tuned), "tuner_trials": len(log),
                               "run_ms": round(run_ms, 3), "replay_ms": round(rep_ms, 3),
                               "gteps_replay": round(arcs / rep_ms / 1e6, 3)}
    # --- A* serving with continuous batching on the 2048x2048 road-like graph ---
    # Poisson arrivals swept over 1k..100k queries/s, slots sized by device memory, the
    # learned policy on (and the fixed automatic Delta as the fallback it replaces).
    from pathfinding_gpu_b200.serving import GpuServer, run_poisson
    from pathfinding_gpu_b200 import policy as P
    road = pf.road(2048, seed=SEED)
    v = pf.uniform_vertices(road.n, 2 * 4000, SEED)
    qs = [(int(v[2 * i]), int(v[2 * i + 1])) for i in range(4000)]
    serving = {"graph": f"road 2048x2048, n={road.n}, m={road.m}", "bucket_drains_per_step": 8}
    from pathfinding_gpu_b200 import Schedule as _Sched
    for mode in ("learned", "fixed", "fixed_warp_drain"):
        opt = (GpuOptions(policy=Policy.Learned) if mode == "learned" else
               GpuOptions(schedule=_Sched.Warp) if mode == "fixed_warp_drain" else GpuOptions())
        with GpuServer(road, slots=0, opt=opt) as srv:
            if mode == "learned" and P.WEIGHTS.exists():
                srv.set_policy(P.load())
            serving["slots"] = srv.slots
            run_poisson(srv, qs[:64], 1000.0, max_rounds=8, seed=2)  # warm
            rates = {}
            for rate in (1000, 2000, 5000, 10000, 20000, 50000, 100000):
                k = min(len(qs), max(1000, rate // 2))
                rep = run_poisson(srv, qs[:k], float(rate), max_rounds=8, seed=3, time_limit_s=20)
                rep.pop("results")
                rates[f"{rate}_qps"] = {kk: (round(x, 3) if isinstance(x, float) else x) for kk, x in rep.items()}
            serving[mode] = rates
    out["serving_road2048"] = serving
    out["extras_wall_s"] = round(time.perf_counter() - t0, 1)
    return out


def run_reference(args):
    """The reference's own cpuMultiSource (OpenMP, every host thread) on the step's full
    batch: the graph is built from the benchmark grid's arcs by the reference's own
    buildCSR, and the sources are the step's; nothing of this repository's engine is
    loaded. Under torchrun only rank 0 runs."""
    if int(os.environ.get("RANK", "0")) != 0:
        return None
    from oracle import oracle as O
    K = args.batch
    n, s, d, w, x, y = O.config_grid_arcs(GRID_SIDE, GRID_SIDE, SEED)
    srcs = O.uniform_vertices(n, K, SEED)
    if O.ref_available():
        R = O.ref_build_csr(n, s, d, w, x, y)
        run = lambda ss: R.multi_source(ss, 0, False)
        threads = O.ref().ref_max_threads()
        kind = "reference"
        m = R.arrays()[5]["m"]
    else:
        g = O.config_grid(GRID_SIDE, GRID_SIDE, SEED)
        run = lambda ss: O.multi_source(g, ss, 0, False)
        threads = O.max_threads()
        kind = "port"
        m = g.m
    for _ in range(args.warmup):
        run(srcs[: max(1, threads)])
    times = []
    for _ in range(args.steps):
        ms, _, _ = run(srcs)
        times.append(ms)
    ms_step = statistics.mean(times)
    m_r = m * K  # the grid is strongly connected: every arc is reachable from every source
    value = m_r / (ms_step * 1e-3) / 1e9
    return {
        "impl": "reference",
        "metric": "GTEPS (reachable arcs / s, SSSP Delta-stepping, batch of sources)",
        "value": round(value, 4), "unit": "GTEPS", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"grid{GRID_SIDE}x{GRID_SIDE} multiSource K={K} Delta-stepping",
                   "n": n, "m": m, "batch": K, "cpu_sources_per_step": K},
        "cpu_baseline": {"value": round(value, 4), "unit": "GTEPS", "cores": int(threads), "kind": kind,
                         "sample": f"all {K} sources of the step, cpuMultiSource OpenMP x{threads}"},
        "e2e": {"value": round(value, 4), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.impl == "reference":
        res = run_reference(args)
        if res is not None:
            print(json.dumps(res))
        return
    D = Dist(args.gpus)
    try:
        res, g, srcs = run_ours(args, D)
        if D.rank == 0:
            if D.world == 1:
                res["cpu_baseline"] = cpu_baseline(g, srcs, min(args.batch, 16))
            if not args.no_extras:
                res["extras"] = extras(g)
            print(json.dumps(res))
    finally:
        D.close()


if __name__ == "__main__":
    main()
