"""ctypes bindings of libpfg_b200.so (the C ABI of include/pfg.h and include/pfg_graphs.h).

The library is built in-tree (python -m pathfinding_gpu_b200.build). There is no
fallback: if the shared object is missing or does not load, every entry point
raises, so a missing extension can never be mistaken for a result.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpfg_b200.so"

u32, u64, i32, f64, f32 = C.c_uint32, C.c_uint64, C.c_int32, C.c_double, C.c_float
P = C.POINTER

PFG_OK = 0
STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "invalid graph", 3: "out of device memory",
    4: "did not converge", 5: "device-side wait timed out", 6: "CUDA error",
    7: "no CUDA device", 8: "capacity exceeded",
}


class PfgOptions(C.Structure):
    _fields_ = [("algo", i32), ("mapping", i32), ("atomic", i32), ("delta", u32),
                ("block_size", i32), ("sync_every", u32), ("compaction", i32), ("policy", i32),
                ("eager", i32), ("blocks_per_sm", i32), ("schedule", i32)]


class PfgStats(C.Structure):
    _fields_ = [("edges_scanned", u64), ("atomics_issued", u64), ("updates", u64), ("pushes", u64),
                ("iterations", u32), ("host_syncs", u32), ("launches", u32), ("buckets", u32),
                ("delta", u32), ("rounds", u32)]


class PfgDeviceInfo(C.Structure):
    _fields_ = [("ok", i32), ("name", C.c_char * 256), ("cc_major", i32), ("cc_minor", i32),
                ("sm_count", i32), ("clock_mhz", i32), ("mem_clock_mhz", i32), ("bus_width", i32),
                ("driver_version", i32), ("runtime_version", i32), ("max_threads_per_sm", i32),
                ("warp_size", i32), ("global_mem", u64), ("shared_per_block", u64),
                ("l2_bytes", u64), ("peak_bandwidth_gbs", f64)]


class PfgTransferStudy(C.Structure):
    _fields_ = [("bytes", f64), ("pageable_ms", f64), ("pinned_ms", f64), ("pinned_streams_ms", f64)]


class PfgGraphInfo(C.Structure):
    _fields_ = [("n", u32), ("m", u32), ("min_w", u32), ("max_w", u32), ("max_deg", u32),
                ("has_xy", i32), ("avg_w", f64), ("avg_deg", f64), ("h_scale", f64)]


class PfgQueryResult(C.Structure):
    _fields_ = [("id", u64), ("src", u32), ("dst", u32), ("dist", u32), ("slot", u32),
                ("submit_us", f64), ("admit_us", f64), ("finish_us", f64)]


# name -> (restype, argtypes); every symbol declared in include/*.h
SIGNATURES = {
    "pfg_server_create": (i32, [P(u32), P(u32), P(u32), P(f64), P(f64), u32, u32, f64, f64, f64, u32,
                                P(PfgOptions), i32, P(C.c_void_p)]),
    "pfg_server_destroy": (None, [C.c_void_p]),
    "pfg_server_submit": (i32, [C.c_void_p, u32, u32, P(u64)]),
    "pfg_server_step": (i32, [C.c_void_p, u32, P(u32), P(u32)]),
    "pfg_server_results": (i32, [C.c_void_p, P(PfgQueryResult), u32, P(u32)]),
    "pfg_server_pending": (u32, [C.c_void_p]),
    "pfg_server_in_flight": (u32, [C.c_void_p]),
    "pfg_server_slots": (u32, [C.c_void_p]),
    "pfg_server_now_us": (f64, [C.c_void_p]),
    "pfg_server_solver": (C.c_void_p, [C.c_void_p]),
    # include/pfg.h
    "pfg_create": (i32, [P(u32), P(u32), P(u32), P(f64), P(f64), u32, u32, f64, f64, f64, u32,
                         P(C.c_void_p)]),
    "pfg_create_on_device": (i32, [P(u32), P(u32), P(u32), P(f64), P(f64), u32, u32, f64, f64, f64,
                                   u32, i32, P(C.c_void_p)]),
    "pfg_destroy": (None, [C.c_void_p]),
    "pfg_upload_ms": (f64, [C.c_void_p]),
    "pfg_device_bytes": (u64, [C.c_void_p]),
    "pfg_auto_delta": (u32, [C.c_void_p]),
    "pfg_num_vertices": (u32, [C.c_void_p]),
    "pfg_max_batch": (u32, [C.c_void_p]),
    "pfg_stream": (C.c_void_p, [C.c_void_p]),
    "pfg_run": (i32, [C.c_void_p, P(u32), u32, i32, u32, P(PfgOptions), P(PfgStats), P(u64), P(f32)]),
    "pfg_run_async": (i32, [C.c_void_p, C.c_void_p, u32, i32, u32, P(PfgOptions)]),
    "pfg_finish": (i32, [C.c_void_p, P(PfgStats)]),
    "pfg_state_device": (C.c_void_p, [C.c_void_p]),
    "pfg_copy_state": (i32, [C.c_void_p, u64, u64, P(u64)]),
    "pfg_copy_dist": (i32, [C.c_void_p, u64, u64, P(u32)]),
    "pfg_run_dist_async": (i32, [C.c_void_p, P(u32), u32, C.POINTER(PfgOptions), P(u32), C.POINTER(PfgStats)]),
    "pfg_dist_wait": (i32, [C.c_void_p, C.POINTER(PfgStats)]),
    "pfg_extract_path": (i32, [C.c_void_p, u32, u32, u32, P(u32), u32, P(u32)]),
    "pfg_query_device": (i32, [i32, P(PfgDeviceInfo)]),
    "pfg_warmup": (i32, []),
    "pfg_transfer_study_run": (i32, [P(u32), P(u32), P(u32), u32, u32, i32, P(PfgTransferStudy)]),
    "pfg_set_policy": (i32, [C.c_void_p, P(f32), u64]),
    "pfg_policy_param_count": (u64, []),
    "pfg_run_traced": (i32, [C.c_void_p, P(u32), u32, P(PfgOptions), P(PfgStats), P(f32), u32, P(u32),
                             P(f32)]),
    "pfg_policy_grad": (i32, [P(f32), P(f32), P(f32), u32, P(f32), P(f32)]),
    "pfg_policy_train": (i32, [P(f32), P(f32), P(f32), u32, u32, f32, P(f32)]),
    "pfg_policy_infer": (i32, [P(f32), P(f32), u32, P(u32)]),
    "pfg_batch_create": (i32, [u32, P(P(u32)), P(P(u32)), P(P(u32)), P(u32), P(u32), u64, u32, i32,
                               P(C.c_void_p)]),
    "pfg_batch_destroy": (None, [C.c_void_p]),
    "pfg_batch_set_instances": (i32, [C.c_void_p, P(u32), P(u32), u32]),
    "pfg_batch_run": (i32, [C.c_void_p, P(PfgOptions), P(PfgStats), P(f32)]),
    "pfg_batch_capture": (i32, [C.c_void_p, P(PfgOptions)]),
    "pfg_batch_replay": (i32, [C.c_void_p, P(PfgStats), P(f32)]),
    "pfg_batch_instance_offset": (u64, [C.c_void_p, u32]),
    "pfg_batch_num_states": (u64, [C.c_void_p]),
    "pfg_batch_copy_state": (i32, [C.c_void_p, u64, u64, P(u64)]),
    "pfg_batch_stream": (C.c_void_p, [C.c_void_p]),
    "pfg_batch_upload_ms": (f64, [C.c_void_p]),
    "pfg_batch_device_bytes": (u64, [C.c_void_p]),
    "pfg_sssp_noalloc": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u32, u32, u32, u32, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "pfg_last_error": (C.c_char_p, []),
    "pfg_status_string": (C.c_char_p, [i32]),
    "pfg_abi_version": (i32, []),
    # include/pfg_graphs.h
    "pfg_graph_from_edges": (i32, [u32, u64, P(u32), P(u32), P(u32), P(f64), P(f64), P(C.c_void_p)]),
    "pfg_graph_from_edges_gpu": (i32, [u32, u64, P(u32), P(u32), P(u32), P(f64), P(f64), i32, P(C.c_void_p)]),
    "pfg_csr_build_device": (i32, [u32, u64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, P(PfgGraphInfo), i32, C.c_void_p]),
    "pfg_graph_gen_grid": (i32, [u32, u32, u64, P(C.c_void_p)]),
    "pfg_graph_gen_rmat": (i32, [u32, u32, f64, f64, f64, u32, u32, u64, P(C.c_void_p)]),
    "pfg_graph_gen_road": (i32, [u32, f64, f64, u32, f64, u64, P(C.c_void_p)]),
    "pfg_graph_union": (i32, [P(C.c_void_p), u32, P(C.c_void_p)]),
    "pfg_graph_load_dimacs": (i32, [C.c_char_p, C.c_char_p, P(C.c_void_p)]),
    "pfg_graph_load_snap": (i32, [C.c_char_p, i32, u32, u64, P(C.c_void_p)]),
    "pfg_graph_save_binary": (i32, [C.c_void_p, C.c_char_p]),
    "pfg_graph_load_binary": (i32, [C.c_char_p, P(C.c_void_p)]),
    "pfg_graph_get_info": (i32, [C.c_void_p, P(PfgGraphInfo)]),
    "pfg_graph_row_offsets": (P(u32), [C.c_void_p]),
    "pfg_graph_col_indices": (P(u32), [C.c_void_p]),
    "pfg_graph_weights": (P(u32), [C.c_void_p]),
    "pfg_graph_x": (P(f64), [C.c_void_p]),
    "pfg_graph_y": (P(f64), [C.c_void_p]),
    "pfg_graph_free": (None, [C.c_void_p]),
    "pfg_graph_pick_sources": (i32, [C.c_void_p, u32, u64, P(u32)]),
}

_lib = None


def load() -> C.CDLL:
    """Loads libpfg_b200.so once; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("PFG_LIB", LIB_PATH))
    if not path.exists():
        raise RuntimeError(f"{path} is missing: build it with `python -m pathfinding_gpu_b200.build`")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class PfgError(RuntimeError):
    """Error raised for a non-zero pfg_status; `status` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int) -> None:
    if status != PFG_OK:
        msg = load().pfg_last_error().decode(errors="replace")
        raise PfgError(status, msg or STATUS_NAMES.get(status, f"status {status}"))


def ptr(arr, ctype):
    """Pointer to a contiguous numpy array (or None)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(P(ctype))
