// pfg_kernels.cu - host-side launch helpers of the persistent SSSP / A* kernel
// and the small utility kernels (padded adjacency build, path and distance
// extraction). The persistent kernel's instantiations are compiled from
// pfg_persistent.cu in separate objects; each object exposes its kernels
// through a getter declared below.
#include "pfg_persistent.cuh"

#include <atomic>
#include <cstdio>

namespace pfg {
// Defined in pfg_persistent.cu, one object per (A*, atomic mode, part):
// part 0 = Thread and Warp mappings (map 0 / 1), part 1 = Hybrid mapping,
// part 2 = Hybrid mapping with warp-worker drains, part 3 = Hybrid mapping with
// independent bucket windows (SSSP only).
#define PFG_DECLARE_GETTERS(A, AM)                        \
    const void* persistent_kernel_##A##_##AM##_0(int map); \
    const void* persistent_kernel_##A##_##AM##_1(int map); \
    const void* persistent_kernel_##A##_##AM##_2(int map);
PFG_DECLARE_GETTERS(0, 0)
PFG_DECLARE_GETTERS(0, 1)
PFG_DECLARE_GETTERS(0, 2)
PFG_DECLARE_GETTERS(1, 0)
PFG_DECLARE_GETTERS(1, 1)
PFG_DECLARE_GETTERS(1, 2)
#undef PFG_DECLARE_GETTERS
const void* persistent_kernel_0_0_3(int map);
const void* persistent_kernel_0_1_3(int map);
const void* persistent_kernel_0_2_3(int map);
}  // namespace pfg

// ===========================================================================
// Host-side launch helpers
// ===========================================================================
namespace pfg {

typedef const void* (*KernelGetter)(int);

// wd: the warp-drain instantiation, iw: the independent-window one (hybrid mapping only).
static const void* kernel_for(bool astar, int am, int map, bool wd = false, bool iw = false) {
    if (am < 0 || am > 2) am = 0;
    if (map < 0 || map > 2) map = 2;
    if (iw && !astar && map == 2) {
        static const KernelGetter iw_table[3] = {persistent_kernel_0_0_3, persistent_kernel_0_1_3,
                                                 persistent_kernel_0_2_3};
        return iw_table[am](map);
    }
    static const KernelGetter table[2][3][3] = {
        {{persistent_kernel_0_0_0, persistent_kernel_0_0_1, persistent_kernel_0_0_2},
         {persistent_kernel_0_1_0, persistent_kernel_0_1_1, persistent_kernel_0_1_2},
         {persistent_kernel_0_2_0, persistent_kernel_0_2_1, persistent_kernel_0_2_2}},
        {{persistent_kernel_1_0_0, persistent_kernel_1_0_1, persistent_kernel_1_0_2},
         {persistent_kernel_1_1_0, persistent_kernel_1_1_1, persistent_kernel_1_1_2},
         {persistent_kernel_1_2_0, persistent_kernel_1_2_1, persistent_kernel_1_2_2}}};
    const int part = map < 2 ? 0 : (wd ? 2 : 1);
    return table[astar ? 1 : 0][am][part](map);
}

// Dynamic shared memory of the persistent kernel (one Coop per CTA); the
// opt-in above 48 KB is set once per instantiation and device (not a stream
// operation, so launches inside a stream capture need nothing more).
static cudaError_t allow_coop_smem(bool astar, int am, int map, bool wd, bool iw = false) {
    static std::atomic<unsigned> done[64];  // bit (iw | wd, astar, am, map) per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const bool w = wd && map == 2;
    const bool v = iw && !astar && map == 2;
    const unsigned bit = 1u << (v ? 27 + am : (w ? 18 : 0) + (astar ? 9 : 0) + 3 * am + map);
    if (dev < 64 && (done[dev].load() & bit)) return cudaSuccess;
    // (room for the independent-window arrays of the largest batch that uses them)
    e = cudaFuncSetAttribute(kernel_for(astar, am, map, w, v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(iw_smem_offset(MAX_BS) + iw_smem_bytes(IW_MAX_INST)));
    if (e == cudaSuccess && dev < 64) done[dev].fetch_or(bit);
    return e;
}

cudaError_t launch_persistent(const RunParams& p, bool astar, int am, int map, int block,
                              int grid, cudaStream_t st) {
    // Cooperative attribute: the driver refuses a grid that cannot be fully
    // resident, which the grid barrier relies on. Also valid in stream capture.
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    if (am < 0 || am > 2) am = 0;
    if (map < 0 || map > 2) map = 2;
    // the warp drain exists for the hybrid mapping only, and its pushes need its kernel
    if (p.warp_drain && map != 2) return cudaErrorInvalidValue;
    const bool wd = p.warp_drain != 0u, iw = p.iw != 0u;
    const void* k = kernel_for(astar, am, map, wd, iw);
    const cudaError_t ea = allow_coop_smem(astar, am, map, wd, iw);
    if (ea != cudaSuccess) return ea;
    if (p.iw && (astar || map != 2 || wd || p.k > IW_MAX_INST)) return cudaErrorInvalidValue;
    cfg.dynamicSmemBytes = p.iw ? iw_smem_offset((u32)block) + iw_smem_bytes(p.k) : coop_bytes((u32)block);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[] = {(void*)&p};
    return cudaLaunchKernelExC(&cfg, k, args);
}

// iw_k > 0: with the independent-window arrays of a run of iw_k instances.
int persistent_blocks_per_sm(bool astar, int am, int map, int block, bool wd, u32 iw_k) {
    int nb = 0;
    if (am < 0 || am > 2) am = 0;
    if (map < 0 || map > 2) map = 2;
    const void* k = kernel_for(astar, am, map, wd, iw_k > 0u);
    const size_t dyn = iw_k ? iw_smem_offset((u32)block) + iw_smem_bytes(iw_k) : coop_bytes((u32)block);
    if (allow_coop_smem(astar, am, map, wd, iw_k > 0u) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, block, dyn) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

// One warp per vertex copies its row into the padded slot.
__global__ void k_build_adj(const u32* __restrict__ row, const u32* __restrict__ col,
                            const u32* __restrict__ w, const u32* __restrict__ prow, u32 n,
                            uint2* __restrict__ adj) {
    const u32 lane = threadIdx.x & 31u;
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 u = warp; u < n; u += nwarps) {
        const u32 r0 = row[u], deg = row[u + 1] - r0;
        const u32 p0 = prow[u], pd = prow[u + 1] - p0;
        for (u32 j = lane; j < pd; j += 32)
            adj[p0 + j] = j < deg ? make_uint2(col[r0 + j], w[r0 + j]) : make_uint2(u, PAD_W);
    }
}

cudaError_t launch_build_adj(const uint32_t* row, const uint32_t* col, const uint32_t* w,
                             const uint32_t* prow, uint32_t n, void* adj, cudaStream_t st) {
    const int bs = 256;
    u32 blocks = (u32)((n + 7u) / 8u);
    if (blocks > 65535u * 4u) blocks = 65535u * 4u;
    if (blocks == 0) blocks = 1;
    k_build_adj<<<blocks, bs, 0, st>>>(row, col, w, prow, n, (uint2*)adj);
    return cudaGetLastError();
}

// Single-thread walk of the parent chain (reference reconstructPath,
// src/cpu_sssp.cpp:124-135): at most n+1 steps, so it always terminates.
__global__ void k_extract_path(const u64* __restrict__ state, u64 base, u32 n, u32 src, u32 dst,
                               u32* __restrict__ path_rev, u32 cap, u32* __restrict__ len) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    u32 v = dst, count = 0;
    for (u64 steps = 0; steps <= n; ++steps) {
        if (count < cap) path_rev[count] = v;
        ++count;
        if (v == src) {
            *len = count <= cap ? count : cap + 1u;
            return;
        }
        const u32 pv = (u32)(__ldcg(state + base + v) & 0xFFFFFFFFull);
        if (pv == NO_PARENT || pv >= n) break;
        v = pv;
    }
    *len = 0;  // broken chain, cycle, or unreachable
}

cudaError_t launch_extract_path(const uint64_t* state, uint64_t base, uint32_t n, uint32_t src,
                                uint32_t dst, uint32_t* path_rev, uint32_t cap, uint32_t* len,
                                cudaStream_t st) {
    k_extract_path<<<1, 32, 0, st>>>(state, base, n, src, dst, path_rev, cap, len);
    return cudaGetLastError();
}

// Distance halves of packed state words, out[i] = state[i] >> 32: the
// reference's per-source distance extraction (src/gpu_sssp.cu:561-565) done
// on the device, so a multi-source result crosses PCIe at 4 bytes per state.
// Bandwidth-bound: 8 bytes read and 4 written per word, 16 words per thread
// in flight per grid-stride pass.
__global__ void k_extract_dist(const u64* __restrict__ state, u64 count, u32* __restrict__ out) {
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = (u32)(__ldcs(state + i) >> 32);
}

cudaError_t launch_extract_dist(const uint64_t* state, uint64_t count, uint32_t* out, int sm_count,
                                cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    const u64 want = (count + 255) / 256;
    const u64 cap = (u64)(sm_count > 0 ? sm_count : 148) * 16;
    k_extract_dist<<<(unsigned)(want < cap ? want : cap), 256, 0, st>>>(state, count, out);
    return cudaGetLastError();
}

}  // namespace pfg
