"""The C ABI library loads and exports every symbol declared in include/*.h (CPU only:
no device compute is called). Also checks the host-only parts of the ABI."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from pathfinding_gpu_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("pfg*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        txt = h.read_text()
        for m in re.finditer(r"PFG_API\s+[\w\s\*]+?\b(pfg_\w+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_headers_declare_the_boundary():
    names = declared_symbols()
    for must in ("pfg_create", "pfg_destroy", "pfg_run", "pfg_last_error", "pfg_query_device",
                 "pfg_transfer_study_run", "pfg_warmup", "pfg_graph_from_edges", "pfg_sssp_noalloc"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = N.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for name in declared_symbols():
        assert hasattr(lib, name)


def test_ctypes_table_covers_every_declared_symbol():
    assert declared_symbols() <= set(N.SIGNATURES), sorted(declared_symbols() - set(N.SIGNATURES))


def test_abi_version_and_status_strings():
    lib = N.load()
    assert lib.pfg_abi_version() == 1
    assert lib.pfg_status_string(0) == b"ok"
    assert lib.pfg_status_string(8) == b"capacity exceeded"


def test_create_rejects_malformed_csr_before_touching_a_gpu():
    import numpy as np
    lib = N.load()
    h = C.c_void_p()

    def create(row, col, w, n, m):
        row = np.asarray(row, np.uint32)
        col = np.asarray(col, np.uint32)
        w = np.asarray(w, np.uint32)
        return lib.pfg_create(N.ptr(row, N.u32), N.ptr(col, N.u32), N.ptr(w, N.u32), None, None, n, m,
                              0.0, 1.0, 1.0, 1, C.byref(h))

    assert create([0, 1, 2], [1, 5], [3, 3], 2, 2) == 2          # col >= n
    assert b"col_indices" in lib.pfg_last_error()
    assert create([0, 2, 2], [1, 1], [5, 3], 2, 2) == 2          # row not sorted by weight
    assert b"not sorted" in lib.pfg_last_error()
    assert create([0, 1, 1], [1], [0], 2, 1) == 2                # zero weight
    assert create([0, 1, 3], [1, 0], [1, 1], 2, 2) == 2          # row_offsets[n] != m
    assert create([0], [], [], 0, 0) == 2                        # no vertices


def test_cpp_dropin_header_is_self_contained(tmp_path):
    # the C++ layer compiles without CUDA headers (the reference's main.cpp is plain C++)
    src = tmp_path / "t.cpp"
    src.write_text('#include "gpu_sssp.h"\nint main(){ GpuOptions o; return o.blockSize == 256 ? 0 : 1; }\n')
    compat = ROOT / "pathfinding_gpu_b200" / "csrc" / "compat"
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", f"-I{ROOT/'include'}", f"-I{compat}", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_streamed_and_copy_entry_points_reject_null_before_touching_a_gpu():
    # argument checks of the distance copy-back and streamed multiSource entry points
    lib = N.load()
    st = N.PfgStats()
    assert lib.pfg_dist_wait(None, C.byref(st)) == 1
    assert b"NULL" in lib.pfg_last_error()
    assert lib.pfg_run_dist_async(None, None, 1, None, None, None) == 1
    assert lib.pfg_copy_dist(None, 0, 1, None) == 1
