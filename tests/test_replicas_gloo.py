"""Replica sharding over a 2-rank gloo process group on CPU (the N > 1 path of bench.py
and pathfinding_gpu_b200.replicas): each rank solves its round-robin shard of the
sources (solve_sharded) and of point-to-point queries (serve_sharded) with the oracle,
and rank 0 must gather exactly the single-process answer."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import pathfinding_gpu_b200 as pf
    from pathfinding_gpu_b200.replicas import ReplicaGroup, serve_sharded, solve_sharded, shard
    from oracle import oracle as O

    g = pf.grid(40, 40, 2026)
    srcs = pf.uniform_vertices(g.n, 7, 99).tolist()
    group = ReplicaGroup(backend="gloo", timeout_s=60)
    assert shard(srcs, rank, world) == srcs[rank::world]

    def solve(mine):
        return np.stack([O.dijkstra(g, s)[0] for s in mine])

    got = solve_sharded(srcs, group, solve)
    pairs = [(int(a), int(b)) for a, b in pf.uniform_vertices(g.n, 2 * 5, 123).reshape(-1, 2)]
    got_pairs = serve_sharded(pairs, group, lambda mine: [int(O.dijkstra(g, s)[0][t]) for s, t in mine])
    mx = group.max(float(rank + 1))
    sm = group.sum(float(rank + 1))
    group.barrier()
    if rank == 0:
        np.savez(out_path, got=got, mx=mx, sm=sm, got_pairs=got_pairs)
    group.close()


def test_two_rank_gloo_replicas(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    out = tmp_path / "res.npz"
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(out))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]

    sys.path.insert(0, str(ROOT))
    import pathfinding_gpu_b200 as pf
    from oracle import oracle as O
    g = pf.grid(40, 40, 2026)
    srcs = pf.uniform_vertices(g.n, 7, 99).tolist()
    want = np.stack([O.dijkstra(g, s)[0] for s in srcs])
    res = np.load(out)
    assert np.array_equal(res["got"], want)
    assert float(res["mx"]) == 2.0 and float(res["sm"]) == 3.0
    pairs = [(int(a), int(b)) for a, b in pf.uniform_vertices(g.n, 2 * 5, 123).reshape(-1, 2)]
    want_pairs = np.array([[O.dijkstra(g, s)[0][t]] for s, t in pairs], np.uint32)
    assert np.array_equal(res["got_pairs"], want_pairs)
