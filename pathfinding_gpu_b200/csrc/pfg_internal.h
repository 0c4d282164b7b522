// pfg_internal.h - host helpers shared by the solver, batch and serving entry
// points of libpfg_b200.so (not part of the C ABI).
#pragma once
#include "../../include/pfg.h"
#include "pfg_common.cuh"

#include <cuda_runtime.h>

namespace pfg {

// Records the calling thread's error message and returns `st`.
pfg_status set_error(pfg_status st, const char* fmt, ...);

// Well-formed CSR with rows sorted by weight and weights in [1, 2^32-2];
// *maxw_out = largest weight.
pfg_status validate_csr(const uint32_t* row, const uint32_t* col, const uint32_t* w, uint32_t n,
                        uint32_t m, u32* maxw_out);

// Round(32 * avgW / avgDeg), at least 1 (reference: src/gpu_sssp.cu:202-206).
u32 auto_delta_of(double avg_w, double avg_deg);

// Engine defaults applied to pfg_options (block size fix-up of the reference,
// src/gpu_sssp.cu:462).
pfg_options default_options();
void sanitize_options(pfg_options& o);

// Launch shape: CTAs per SM for the persistent kernel.
int blocks_per_sm_for(const pfg_options& o, bool astar, int map);

// Eager sub-rounds when the caller leaves the choice to the engine.
u32 eager_rounds_for(const pfg_options& o);

// Milliseconds from the PFG_TIMEOUT_MS environment variable (default 2000)
// as the bound of every device-side wait, in nanoseconds.
u64 device_timeout_ns();

}  // namespace pfg
