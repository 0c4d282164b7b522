"""B200-native SSSP / A* engine: hand-written sm_100a kernels behind the reference's
GpuSolver interface (C ABI: include/pfg.h; C++: include/gpu_sssp.h; Python: this package)."""
from .graphs import (CSRGraph, buildCSR, grid, rmat, road, grid_batch, grid_batch_sides, union,
                     load_dimacs, load_snap, load_binary, pick_sources, uniform_vertices, SplitMix64,
                     DEFAULT_SEED)
from .solver import (GpuSolver, GpuOptions, GpuStats, GpuRunResult, GpuAlgo, Mapping, AtomicMode,
                     Compaction, Policy, Schedule, INF_DIST, NO_PARENT, unpack, reconstruct_path, device_info)
from ._native import PfgError

__all__ = [
    "CSRGraph", "buildCSR", "grid", "rmat", "road", "grid_batch", "grid_batch_sides", "union",
    "load_dimacs", "load_snap", "load_binary", "pick_sources", "uniform_vertices", "SplitMix64",
    "DEFAULT_SEED", "GpuSolver", "GpuOptions", "GpuStats", "GpuRunResult", "GpuAlgo", "Mapping",
    "AtomicMode", "Compaction", "Policy", "Schedule", "INF_DIST", "NO_PARENT", "unpack", "reconstruct_path",
    "device_info", "PfgError",
]
