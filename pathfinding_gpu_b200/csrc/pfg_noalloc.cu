// pfg_noalloc.cu - SSSP entry point that allocates no memory.
//
// Some callers must not allocate device memory at run time: a host
// application or framework that owns every byte of device memory through
// its own pool (a plugin may only use the buffers it is handed), code on a
// latency budget that cannot afford cudaMalloc's implicit synchronisation
// and fragmentation, or a process that has reserved the whole GPU before
// this library runs. For them, pfg_sssp_noalloc runs the same persistent
// Delta-stepping kernel as pfg_run, on CSR arrays and an output buffer the
// caller already has in device memory, with all of the kernel's scratch
// (padded adjacency, queues, dedup stamps, control block) in one fixed
// file-scope device array. Nothing is allocated per call: no cudaMalloc,
// no cudaFree, no allocating library routine.
//
// The array's size is fixed at build time (kScratchBytes, about 7.6 MB);
// every GPU on which this library's module is loaded holds it until the
// process exits. Graphs larger than the limits below are rejected.
#include "../../include/pfg.h"
#include "pfg_common.cuh"
#include "pfg_internal.h"
#include "pfg_kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

using namespace pfg;

extern "C" void pfg_internal_set_error(const char* msg);

namespace {

// Limits of the fixed scratch array.
constexpr u32 kMaxVertices = PFG_NOALLOC_MAX_VERTICES;
constexpr u32 kMaxPaddedArcs = PFG_NOALLOC_MAX_ARCS;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffCtl = 0;
constexpr size_t kOffSrc = align256(kOffCtl + sizeof(Ctl));
constexpr size_t kOffProw = align256(kOffSrc + 16);
constexpr size_t kOffAdj = align256(kOffProw + ((size_t)kMaxVertices + 1) * 4);
constexpr size_t kOffQueues = align256(kOffAdj + (size_t)kMaxPaddedArcs * 8);
constexpr size_t kOffStamps = align256(kOffQueues + 5 * (size_t)kMaxVertices * 4);
constexpr size_t kScratchBytes = align256(kOffStamps + 3 * (size_t)kMaxVertices * 4);

// The scratch. In host code this name is only a stand-in for the symbol: its
// device address comes from cudaGetSymbolAddress (see scratch_on_current_device).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_dev_scratch[kMaxDevices] = {};
int g_dev_sms[kMaxDevices] = {};
int g_dev_bps[kMaxDevices] = {};

pfg_status na_fail(pfg_status st, const char* msg) {
    pfg_internal_set_error(msg);
    return st;
}

// Failed device-side checks of the caller's CSR (bits of the error word in
// the scratch, reported in d_status_out[1]).
constexpr u32 kBadRows = 1u;       // row_offsets[0] != 0, row_offsets[n] != m, or a decreasing offset
constexpr u32 kBadCapacity = 2u;   // the rows padded to 4 arcs do not fit the scratch
constexpr u32 kBadColumn = 4u;     // col_indices[k] >= n
constexpr u32 kBadWeight = 8u;     // weights[k] == 0 or 2^32 - 1
constexpr u32 kBadOrder = 16u;     // a row is not sorted by weight

// Checks the row offsets and writes the padded row starts (rows rounded up to
// 4 arcs), by one CTA of 1024 threads. Nothing is written to prow when a check
// fails: the error word is set and the later kernels of the call leave the
// scratch alone, so a malformed CSR cannot make any kernel of this call write
// outside the scratch or the caller's output.
__global__ void k_na_pad_rows(const u32* __restrict__ row, u32 n, u32 m, u32* __restrict__ prow,
                              u32* __restrict__ err) {
    __shared__ unsigned long long part[1024];
    __shared__ u32 s_bad;
    const u32 t = threadIdx.x, T = blockDim.x;
    if (t == 0) s_bad = 0u;
    __syncthreads();
    const u32 per = (n + T - 1) / T;
    const u32 b = min(n, t * per), e = min(n, b + per);
    unsigned long long sum = 0;
    u32 bad = 0;
    for (u32 u = b; u < e; ++u) {
        const u32 r0 = row[u], r1 = row[u + 1];
        if (r1 < r0) bad |= kBadRows;
        else sum += (r1 - r0 + ROW_ALIGN - 1) / ROW_ALIGN * ROW_ALIGN;
    }
    if (t == 0 && (row[0] != 0u || row[n] != m)) bad |= kBadRows;
    if (bad) atomicOr(&s_bad, bad);
    part[t] = sum;
    __syncthreads();
    if (t == 0) {  // n <= 65536: a serial pass over T partial sums is cheap
        unsigned long long acc = 0;
        for (u32 i = 0; i < T; ++i) {
            const unsigned long long v = part[i];
            part[i] = acc;
            acc += v;
        }
        if (acc > kMaxPaddedArcs) s_bad |= kBadCapacity;
        *err = s_bad;
        if (!s_bad) prow[n] = (u32)acc;
    }
    __syncthreads();
    if (s_bad) return;  // block-uniform
    u32 acc = (u32)part[t];
    for (u32 u = b; u < e; ++u) {
        prow[u] = acc;
        acc += (row[u + 1] - row[u] + ROW_ALIGN - 1) / ROW_ALIGN * ROW_ALIGN;
    }
}

// One warp per vertex copies its row into the padded slot, checking every arc:
// a column >= n or a weight outside [1, 2^32 - 2] is replaced by a padding arc
// (so the relaxation could never leave the state array) and, like a row that
// is not sorted by weight, sets the error word, which cancels the run. Does
// nothing when the row offsets failed their checks.
__global__ void k_na_build_adj(const u32* __restrict__ row, const u32* __restrict__ col,
                               const u32* __restrict__ w, const u32* __restrict__ prow, u32 n,
                               uint2* __restrict__ adj, u32* __restrict__ err) {
    if (*(volatile u32*)err) return;  // written by k_na_pad_rows, earlier on the same stream
    const u32 lane = threadIdx.x & 31u;
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    u32 bad = 0;
    for (u32 u = warp; u < n; u += nwarps) {
        const u32 r0 = row[u], deg = row[u + 1] - r0;
        const u32 p0 = prow[u], pd = prow[u + 1] - p0;  // pd >= deg: rows were checked
        for (u32 j = lane; j < pd; j += 32) {
            uint2 a = make_uint2(u, PAD_W);
            if (j < deg) {
                const u32 c = col[r0 + j], ww = w[r0 + j];
                if (c >= n) bad |= kBadColumn;
                else if (ww == 0u || ww == PAD_W) bad |= kBadWeight;
                else a = make_uint2(c, ww);
                if (j > 0 && w[r0 + j - 1] > ww) bad |= kBadOrder;
            }
            adj[p0 + j] = a;
        }
    }
    if (bad) atomicOr(err, bad);
}

// Control block of one run; the persistent epoch counters restart at 0 because
// the stamp words were just cleared.
// A failed CSR check (error word != 0) starts the run with a bad-graph status:
// the persistent kernel then only initialises the output and stops.
__global__ void k_na_init(Ctl* ctl, u32* src_slot, const u32* err, u32 src, u32 delta, u32 round_cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Ctl c;
    memset(&c, 0, sizeof(c));
    c.rd.phase = PH_INIT;
    c.rd.status = *err ? (u32)DS_BAD_GRAPH : (u32)DS_OK;
    c.rd.delta = delta;
    c.rd.heavy = 1u;  // the largest weight is not known here; the light/heavy split handles any Delta
    c.rd.map_mode = 1u;
    c.far_min[0] = c.far_min[1] = ~0ull;
    c.round_cap = round_cap;
    c.delta0 = delta;
    *ctl = c;
    *src_slot = src;
}

// Copies the outcome of the run into the caller's status words:
// [0] pfg_status of the run, [1] device rounds, [2] buckets, [3] non-empty rounds;
// for a graph that failed the device-side checks [0] is PFG_ERR_INVALID_GRAPH
// (PFG_ERR_CAPACITY when its padded rows do not fit the scratch), [1] the mask
// of failed checks and [2], [3] zero.
__global__ void k_na_status(const Ctl* ctl, const u32* err, u32* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const u32 bad = *err;
    if (bad) {
        out[0] = (bad & kBadCapacity) ? (u32)PFG_ERR_CAPACITY : (u32)PFG_ERR_INVALID_GRAPH;
        out[1] = bad;
        out[2] = out[3] = 0u;
        return;
    }
    const u32 ds = ctl->rd.status;
    out[0] = ds == DS_OK ? (u32)PFG_OK
           : ds == DS_BAD_SOURCE ? (u32)PFG_ERR_INVALID_ARGUMENT
           : ds == DS_NOT_CONVERGED ? (u32)PFG_ERR_NOT_CONVERGED
           : ds == DS_TIMEOUT ? (u32)PFG_ERR_DEVICE_TIMEOUT : (u32)PFG_ERR_CUDA;
    out[1] = ctl->rounds;
    out[2] = ctl->buckets;
    out[3] = ctl->iterations;
}

// Device address of the scratch array on the current device. The first call
// on each device looks the symbol up (this also loads the module on that
// device); later calls reuse the cached address.
pfg_status scratch_on_current_device(int* dev_out, unsigned char** ptr_out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return na_fail(PFG_ERR_NO_DEVICE, "pfg_sssp_noalloc: no current CUDA device");
    }
    if (dev < 0 || dev >= kMaxDevices) return na_fail(PFG_ERR_NO_DEVICE, "pfg_sssp_noalloc: device ordinal too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_dev_scratch[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            char buf[256];
            snprintf(buf, sizeof(buf), "pfg_sssp_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return na_fail(PFG_ERR_CUDA, buf);
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            return na_fail(PFG_ERR_CUDA, "pfg_sssp_noalloc: cannot read the SM count");
        }
        const int bps = persistent_blocks_per_sm(false, 0, PFG_MAP_HYBRID, 1024);
        if (bps <= 0) return na_fail(PFG_ERR_CUDA, "pfg_sssp_noalloc: occupancy query failed");
        g_dev_sms[dev] = sms;
        g_dev_bps[dev] = bps;
        g_dev_scratch[dev] = (unsigned char*)p;
    }
    *dev_out = dev;
    *ptr_out = g_dev_scratch[dev];
    return PFG_OK;
}

}  // namespace

extern "C" pfg_status pfg_sssp_noalloc(const uint32_t* d_row_offsets, const uint32_t* d_col_indices,
                                       const uint32_t* d_weights, uint32_t n, uint32_t m,
                                       uint32_t src, uint32_t delta, uint64_t* d_state_out,
                                       uint32_t* d_status_out, void* stream) {
    if (!d_row_offsets || (m > 0 && (!d_col_indices || !d_weights)) || !d_state_out || !d_status_out)
        return na_fail(PFG_ERR_INVALID_ARGUMENT, "pfg_sssp_noalloc: NULL device pointer");
    if (n == 0) return na_fail(PFG_ERR_INVALID_GRAPH, "pfg_sssp_noalloc: graph has no vertices");
    if (n > kMaxVertices) {
        char buf[200];
        snprintf(buf, sizeof(buf), "pfg_sssp_noalloc: n = %u exceeds the fixed scratch limit of %u vertices", n,
                 kMaxVertices);
        return na_fail(PFG_ERR_CAPACITY, buf);
    }
    if ((uint64_t)m + 3ull * n > kMaxPaddedArcs) {
        char buf[200];
        snprintf(buf, sizeof(buf),
                 "pfg_sssp_noalloc: m + 3n = %llu exceeds the fixed scratch limit of %u padded arcs",
                 (unsigned long long)m + 3ull * n, kMaxPaddedArcs);
        return na_fail(PFG_ERR_CAPACITY, buf);
    }
    if (src >= n) return na_fail(PFG_ERR_INVALID_ARGUMENT, "pfg_sssp_noalloc: source out of range");
    if (delta == 0) return na_fail(PFG_ERR_INVALID_ARGUMENT, "pfg_sssp_noalloc: delta must be >= 1");

    int dev = 0;
    unsigned char* base = nullptr;
    pfg_status st = scratch_on_current_device(&dev, &base);
    if (st != PFG_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;

    Ctl* ctl = (Ctl*)(base + kOffCtl);
    u32* src_slot = (u32*)(base + kOffSrc);
    u32* err = src_slot + 1;  // failed CSR checks of this call (bits kBad*)
    u32* prow = (u32*)(base + kOffProw);
    uint2* adj = (uint2*)(base + kOffAdj);
    u32* q = (u32*)(base + kOffQueues);
    u32* stamps = (u32*)(base + kOffStamps);

    // The stamp words must start at zero (their epochs restart with the control block).
    cudaError_t e = cudaMemsetAsync(stamps, 0, 3 * (size_t)n * 4, s);
    if (e == cudaSuccess) {
        k_na_pad_rows<<<1, 1024, 0, s>>>(d_row_offsets, n, m, prow, err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        const u32 blocks = std::max<u32>(1u, std::min<u32>((n + 7u) / 8u, 4096u));
        k_na_build_adj<<<blocks, 256, 0, s>>>(d_row_offsets, d_col_indices, d_weights, prow, n, adj, err);
        e = cudaGetLastError();
    }
    const u32 round_cap = (u32)std::min<unsigned long long>(4ull * n + 1000ull, 0x7FFFFFFFull);
    if (e == cudaSuccess) {
        k_na_init<<<1, 1, 0, s>>>(ctl, src_slot, err, src, delta, round_cap);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        RunParams p;
        memset(&p, 0, sizeof(p));
        p.adj = adj;
        p.prow = prow;
        p.n = n;
        p.maxw = 0xFFFFFFFEu;  // unknown here: keep every arc eligible for the heavy pass
        p.m = m;
        p.k = 1;
        p.total = n;
        p.srcs = src_slot;
        p.state = d_state_out;
        p.nearq[0] = q;
        p.nearq[1] = q + kMaxVertices;
        p.farq[0] = q + 2 * (size_t)kMaxVertices;
        p.farq[1] = q + 3 * (size_t)kMaxVertices;
        p.rq = q + 4 * (size_t)kMaxVertices;
        p.near_stamp = stamps;
        p.far_stamp = stamps + n;
        p.r_stamp = stamps + 2 * (size_t)n;
        p.ctl = ctl;
        p.delta = delta;
        p.mode = MODE_DELTA;
        // the engine defaults of pfg_run: eager sub-rounds on low-degree graphs
        // only, the PFG_TIMEOUT_MS bound on every device-side wait
        p.eager = (double)m / (double)n > kEagerMaxAvgDegree ? 0u : kDefaultEager;
        const int grid = g_dev_sms[dev] * g_dev_bps[dev];
        p.eager_max_items = (u32)std::max(1, grid * 1024 / 4);
        p.timeout_ns = device_timeout_ns();
        e = launch_persistent(p, false, PFG_ATOMIC_MIN_RBA, PFG_MAP_HYBRID, 1024, grid, s);
    }
    if (e == cudaSuccess) {
        k_na_status<<<1, 1, 0, s>>>(ctl, err, d_status_out);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        char buf[256];
        snprintf(buf, sizeof(buf), "pfg_sssp_noalloc: launch failed: %s", cudaGetErrorString(e));
        return na_fail(PFG_ERR_CUDA, buf);
    }
    return PFG_OK;
}
