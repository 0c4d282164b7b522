"""Build recipe of libpfg_b200.so (CUDA kernels + C ABI), compiled in-tree for sm_100a.

Usage: python -m pathfinding_gpu_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libpfg_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fvisibility=hidden",
    "-I", str(ROOT / "include"),
]
SOURCES = ["pfg_kernels.cu", "pfg_solver.cu", "pfg_device.cu", "pfg_policy.cu", "pfg_batch.cu",
           "pfg_serve.cu", "pfg_noalloc.cu", "pfg_csr.cu", "pfg_graphs.cpp"]
HEADERS = ["pfg_common.cuh", "pfg_kernels.h", "pfg_internal.h", "pfg_persistent.cuh"]
# The persistent kernel's instantiations, one object per (A*, atomic mode, part):
# compiled from one source in parallel (each instantiation is a large fully inlined kernel).
PERSISTENT = "pfg_persistent.cu"
VARIANTS = [(a, am, part) for a in (0, 1) for am in (0, 1, 2) for part in (0, 1, 2)] + \
           [(0, am, 3) for am in (0, 1, 2)]  # part 3: independent bucket windows (SSSP only)


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every source for sm_100a and links libpfg_b200.so in the package directory."""
    OBJ.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = [CSRC / h for h in HEADERS] + list((ROOT / "include").glob("*.h"))
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    jobs = []
    objs = []
    for src in srcs:
        obj = OBJ / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
            if src.suffix == ".cpp":
                cmd = [nvcc] + NVCC_FLAGS + ["-x", "c++", "-c", str(src), "-o", str(obj)]
            jobs.append((src, cmd))
    psrc = CSRC / PERSISTENT
    for a, am, part in VARIANTS:
        obj = OBJ / f"pfg_persistent_{a}_{am}_{part}.o"
        objs.append(obj)
        if force or _stale(obj, [psrc] + headers):
            defs = [f"-DPFG_V_ASTAR={a}", f"-DPFG_V_AM={am}", f"-DPFG_V_PART={part}"]
            jobs.append((psrc, [nvcc] + NVCC_FLAGS + defs + ["-c", str(psrc), "-o", str(obj)]))
    # the slowest objects first
    jobs.sort(key=lambda j: 0 if j[0].name == PERSISTENT else 1)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(max(os.cpu_count() or 8, 8), len(jobs))) as ex:
            futs = {ex.submit(subprocess.run, cmd, capture_output=True, text=True): src for src, cmd in jobs}
            for fut in cf.as_completed(futs):
                r = fut.result()
                if verbose and r.stdout:
                    print(r.stdout)
                if r.returncode != 0:
                    raise RuntimeError(f"nvcc failed on {futs[fut].name}:\n{r.stderr}")
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
