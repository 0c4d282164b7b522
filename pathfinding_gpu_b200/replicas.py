"""Multi-GPU replicas: one process per GPU, the whole graph on every GPU, queries sharded.

A single SSSP does not shard across GPUs at these sizes (it would need an
all-to-all of remote relaxations on every round), so the multi-GPU form is data
parallel over independent queries: rank r solves sources r, r+W, r+2W, ... on
its own GPU (serve_sharded: point-to-point queries r, r+W, ... on its own
serving engine) and the per-query results are gathered on rank 0. There is no
collective on the data path; the process group only carries barriers, timing
reductions and the final gather (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def shard(items: Sequence, rank: int, world: int) -> list:
    """Round-robin shard of `items` owned by `rank`."""
    return [items[i] for i in range(rank, len(items), world)]


class ReplicaGroup:
    """Process group of the replicas (env: RANK, WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT)."""

    def __init__(self, backend: Optional[str] = None, timeout_s: int = 120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = torch.device("cuda", self.local)
                kw["device_id"] = self.device
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            self.dist = dist
            self.backend = backend

    def _tensor(self, values):
        import torch
        t = torch.tensor(values, dtype=torch.float64)
        return t.to(self.device) if self.device is not None else t

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        t = self._tensor([x])
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return x
        t = self._tensor([x])
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def gather_rows(self, rows: np.ndarray, total: int) -> Optional[np.ndarray]:
        """Gathers each rank's round-robin shard of a [total, width] array on rank 0."""
        if not self.dist:
            return rows
        import torch
        width = rows.shape[1] if rows.ndim == 2 else 0
        per = (total + self.world - 1) // self.world
        buf = np.zeros((per, width), rows.dtype)
        buf[: rows.shape[0]] = rows
        t = torch.from_numpy(buf.astype(np.int64))
        if self.device is not None:
            t = t.to(self.device)
        parts = [torch.empty_like(t) for _ in range(self.world)] if self.rank == 0 else None
        self.dist.gather(t, parts, dst=0)
        if self.rank != 0:
            return None
        out = np.zeros((total, width), rows.dtype)
        for r, part in enumerate(parts):
            idx = list(range(r, total, self.world))
            out[idx] = part.cpu().numpy()[: len(idx)].astype(rows.dtype)
        return out

    def close(self) -> None:
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None


def serve_sharded(pairs: Sequence[Tuple[int, int]], group: ReplicaGroup,
                  answer: Callable[[List[Tuple[int, int]]], Sequence[int]]) -> Optional[np.ndarray]:
    """Point-to-point queries sharded round-robin over the replicas: each rank
    answers its shard with `answer` (pairs -> target distances; on a GPU, its own
    GpuServer through serving.answer_all) and rank 0 gathers the distances in
    query order (None on the other ranks)."""
    mine = shard(list(pairs), group.rank, group.world)
    d = np.asarray(answer(mine) if mine else [], np.uint32).reshape(-1, 1)
    return group.gather_rows(d, len(pairs))


def solve_sharded(sources: Sequence[int], group: ReplicaGroup,
                  solve: Callable[[List[int]], np.ndarray]) -> Optional[np.ndarray]:
    """Runs `solve` (sources -> [k, n] distances) on this rank's shard and gathers
    every source's row on rank 0 (None on the other ranks)."""
    mine = shard(list(sources), group.rank, group.world)
    rows = solve(mine) if mine else None
    if rows is None:
        rows = np.zeros((0, 0), np.uint32)
    n = rows.shape[1] if rows.size else 0
    if group.world > 1:
        n = int(group.max(float(n)))
        if rows.size == 0:
            rows = np.zeros((0, n), np.uint32)
    return group.gather_rows(rows, len(sources))
