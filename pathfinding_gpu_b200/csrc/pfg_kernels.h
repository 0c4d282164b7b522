// pfg_kernels.h - host entry points of the device kernels (no CUDA types
// leak past the C ABI; this header is internal to libpfg_b200.so).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pfg {

struct RunParams;

// Persistent relaxation kernel: one cooperative launch runs a whole query.
// astar / am (atomic mode 0..2) / map (mapping 0..2) select the instantiation.
cudaError_t launch_persistent(const RunParams& p, bool astar, int am, int map, int block,
                              int grid, cudaStream_t st);
// Largest number of co-resident CTAs per SM for that instantiation (0 on error);
// wd: the warp-drain instantiation (hybrid mapping).
int persistent_blocks_per_sm(bool astar, int am, int map, int block, bool wd = false, u32 iw_k = 0);

// Builds the padded interleaved adjacency adj[prow[u] ..] from a plain CSR.
cudaError_t launch_build_adj(const uint32_t* row, const uint32_t* col, const uint32_t* w,
                             const uint32_t* prow, uint32_t n, void* adj, cudaStream_t st);

// Follows parent pointers of state[base .. base+n) from dst back to src and
// writes the reversed chain to path_rev; *len = number of vertices (0 when the
// chain is broken or dst is unreachable), or cap+1 when it does not fit.
cudaError_t launch_extract_path(const uint64_t* state, uint64_t base, uint32_t n,
                                uint32_t src, uint32_t dst, uint32_t* path_rev, uint32_t cap,
                                uint32_t* len, cudaStream_t st);

// out[i] = distance half of state[i] for i < count (grid of at most 16 CTAs per SM).
cudaError_t launch_extract_dist(const uint64_t* state, uint64_t count, uint32_t* out, int sm_count,
                                cudaStream_t st);

}  // namespace pfg
