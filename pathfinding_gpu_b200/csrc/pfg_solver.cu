// pfg_solver.cu - host orchestration and C ABI of the B200 SSSP / A* engine.
//
// Replaces the reference's GpuSolver::Impl (src/gpu_sssp.cu:61-534): one-time
// device allocation and CSR upload, then one persistent cooperative launch per
// query. Errors are reported as pfg_status codes plus a thread-local message
// instead of exit() (reference: src/cuda_check.cuh:9-17) and exceptions.
#include "../../include/pfg.h"
#include "pfg_common.cuh"
#include "pfg_kernels.h"
#include "pfg_internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace pfg;

// ---------------------------------------------------------------------------
// Error handling
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

static pfg_status fail(pfg_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

pfg_status pfg::set_error(pfg_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

#define PFG_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e__ = (call);                                                        \
        if (e__ != cudaSuccess) {                                                        \
            const pfg_status st__ = e__ == cudaErrorMemoryAllocation ? PFG_ERR_OUT_OF_MEMORY \
                                                                     : PFG_ERR_CUDA;     \
            cudaGetLastError();                                                          \
            return fail(st__, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e__),   \
                        __FILE__, __LINE__);                                             \
        }                                                                                \
    } while (0)

extern "C" const char* pfg_last_error(void) { return g_last_error.c_str(); }
extern "C" void pfg_internal_set_error(const char* msg) { g_last_error = msg ? msg : ""; }
extern "C" int32_t pfg_abi_version(void) { return PFG_ABI_VERSION; }
extern "C" const char* pfg_status_string(pfg_status st) {
    switch (st) {
        case PFG_OK: return "ok";
        case PFG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PFG_ERR_INVALID_GRAPH: return "invalid graph";
        case PFG_ERR_OUT_OF_MEMORY: return "out of device memory";
        case PFG_ERR_NOT_CONVERGED: return "did not converge";
        case PFG_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case PFG_ERR_CUDA: return "CUDA error";
        case PFG_ERR_NO_DEVICE: return "no CUDA device";
        case PFG_ERR_CAPACITY: return "capacity exceeded";
    }
    return "unknown status";
}

// ---------------------------------------------------------------------------
// Solver object
// ---------------------------------------------------------------------------
// struct pfg_solver is defined in pfg_internal.h (shared with the serving engine).

u32 pfg::auto_delta_of(double avg_w, double avg_deg) {
    // Davidson et al.: Delta ~ warp size * average weight / average degree
    // (reference: src/gpu_sssp.cu:202-206).
    const double d = 32.0 * avg_w / std::max(1.0, avg_deg);
    const long long r = std::llround(d);
    return (u32)std::max<long long>(1, std::min<long long>(r, 0x7FFFFFFFll));
}

static void destroy_solver(pfg_solver* s) {
    if (!s) return;
    if (s->device >= 0) cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    for (void* p : s->allocs) cudaFree(p);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->h_srcs) cudaFreeHost(s->h_srcs);
    if (s->d_trace) cudaFree(s->d_trace);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->ev_split) cudaEventDestroy(s->ev_split);
    if (s->ev_copied) cudaEventDestroy(s->ev_copied);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
    cudaGetLastError();
    delete s;
}

pfg_status pfg::validate_csr(const uint32_t* row, const uint32_t* col, const uint32_t* w,
                               uint32_t n, uint32_t m, u32* maxw_out) {
    if (n == 0) return fail(PFG_ERR_INVALID_GRAPH, "graph has no vertices");
    if (!row || (m > 0 && (!col || !w)))
        return fail(PFG_ERR_INVALID_GRAPH, "CSR arrays must not be NULL");
    if (row[0] != 0) return fail(PFG_ERR_INVALID_GRAPH, "row_offsets[0] must be 0");
    if (row[n] != m) return fail(PFG_ERR_INVALID_GRAPH, "row_offsets[n] = %u but m = %u", row[n], m);
    u32 maxw = 0;
    for (u32 u = 0; u < n; ++u) {
        const u32 b = row[u], e = row[u + 1];
        if (e < b) return fail(PFG_ERR_INVALID_GRAPH, "row_offsets decreases at vertex %u", u);
        for (u32 k = b; k < e; ++k) {
            if (col[k] >= n) return fail(PFG_ERR_INVALID_GRAPH, "col_indices[%u] = %u >= n", k, col[k]);
            if (w[k] == 0 || w[k] == PAD_W)
                return fail(PFG_ERR_INVALID_GRAPH, "weights[%u] = %u outside [1, 2^32-2]", k, w[k]);
            if (k > b && w[k] < w[k - 1])
                return fail(PFG_ERR_INVALID_GRAPH,
                            "row %u is not sorted by weight (arc %u); build the CSR with rows "
                            "sorted by (w, dst)", u, k);
            maxw = std::max(maxw, w[k]);
        }
    }
    *maxw_out = maxw;
    return PFG_OK;
}

extern "C" pfg_status pfg_create_on_device(const uint32_t* row, const uint32_t* col,
                                           const uint32_t* w, const double* x, const double* y,
                                           uint32_t n, uint32_t m, double h_scale, double avg_w,
                                           double avg_deg, uint32_t max_batch, int32_t device,
                                           pfg_solver** out) {
    if (!out) return fail(PFG_ERR_INVALID_ARGUMENT, "out must not be NULL");
    *out = nullptr;
    if ((x == nullptr) != (y == nullptr))
        return fail(PFG_ERR_INVALID_ARGUMENT, "x and y must both be set or both be NULL");
    u32 maxw = 0;
    pfg_status st = validate_csr(row, col, w, n, m, &maxw);
    if (st != PFG_OK) return st;
    const u32 K = std::max<u32>(1, max_batch);
    if ((u64)K * n >= 0xFFFFFFFFull)
        return fail(PFG_ERR_INVALID_ARGUMENT, "maxBatch * n must be < 2^32");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) {
        cudaGetLastError();
        return fail(PFG_ERR_NO_DEVICE, "CUDA device %d not available", device);
    }

    // Padded row starts: each row rounded up to a multiple of 4 arcs; when no
    // row has more than 4 arcs (grid-like graphs), every row gets exactly 4
    // slots, so row u starts at 4u and the kernel needs no prow load.
    std::vector<u32> prow((size_t)n + 1);
    u64 acc = 0;
    u32 max_deg = 0;
    u64 hub_rows = 0;  // rows long enough to be hubs for the smallest CTA (8 x 32 arcs)
    for (u32 u = 0; u < n; ++u) {
        const u32 deg = row[u + 1] - row[u];
        max_deg = std::max(max_deg, deg);
        hub_rows += deg > 256u ? 1u : 0u;
    }
    const bool uniform_rows = max_deg <= ROW_ALIGN;
    for (u32 u = 0; u < n; ++u) {
        prow[u] = (u32)acc;
        const u32 deg = row[u + 1] - row[u];
        acc += uniform_rows ? ROW_ALIGN : (u64)((deg + ROW_ALIGN - 1) / ROW_ALIGN) * ROW_ALIGN;
        if (acc >= 0xFFFFFFF0ull) return fail(PFG_ERR_INVALID_GRAPH, "padded arc count exceeds 2^32");
    }
    prow[n] = (u32)acc;

    pfg_solver* s = new pfg_solver();
    s->device = device;
    s->n = n;
    s->m = m;
    s->K = K;
    s->maxw = maxw;
    s->max_deg = max_deg;
    s->row_stride = uniform_rows ? ROW_ALIGN : 0u;
    s->hub_rows = hub_rows;
    s->m_pad = acc;
    s->hscale = h_scale;
    s->avg_w = avg_w;
    s->avg_deg = avg_deg;
    s->has_xy = x != nullptr;
    auto bail = [&](pfg_status e) {
        destroy_solver(s);
        return e;
    };
#define TRY(expr)                                   \
    do {                                            \
        pfg_status e_ = (expr);                     \
        if (e_ != PFG_OK) return bail(e_);          \
    } while (0)
#define TRYC(call)                                                                          \
    do {                                                                                    \
        cudaError_t e__ = (call);                                                           \
        if (e__ != cudaSuccess) {                                                           \
            cudaGetLastError();                                                             \
            return bail(fail(e__ == cudaErrorMemoryAllocation ? PFG_ERR_OUT_OF_MEMORY       \
                                                              : PFG_ERR_CUDA,               \
                             "%s failed: %s", #call, cudaGetErrorString(e__)));            \
        }                                                                                   \
    } while (0)

    TRYC(cudaSetDevice(device));
    TRYC(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device));
    int coop = 0;
    TRYC(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    if (!coop) return bail(fail(PFG_ERR_NO_DEVICE, "device %d lacks cooperative launch", device));

    // Memory precheck (reference: src/gpu_sssp.cu:113-127).
    const u64 Kn = (u64)K * n;
    const u64 need = s->m_pad * 8 + (u64)(n + 1) * 4 + (s->has_xy ? (u64)n * 16 : 0) + Kn * 8 +
                     5 * Kn * 4 + 3 * Kn * 4 + 2 * ((u64)n / 32 + 1) * 4 + (u64)(n + 1) * 4 +
                     ((u64)n + 1) * 4 + 2 * (u64)m * 4;  // last term: upload staging on device
    size_t free_b = 0, total_b = 0;
    TRYC(cudaMemGetInfo(&free_b, &total_b));
    if (need > free_b)
        return bail(fail(PFG_ERR_OUT_OF_MEMORY,
                         "Not enough GPU memory: need %.1f MB, free %.1f MB (reduce graph or batch)",
                         need / 1048576.0, free_b / 1048576.0));

    TRYC(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    TRYC(cudaEventCreate(&s->ev0));
    TRYC(cudaEventCreate(&s->ev1));

    // ---- upload: pinned staging, three streams (reference: src/gpu_sssp.cu:138-152),
    //      then the padded adjacency is built on the device ----
    auto t0 = std::chrono::steady_clock::now();
    TRY(s->dalloc(&s->d_adj, s->m_pad));
    TRY(s->dalloc(&s->d_prow, (u64)n + 1));
    {
        u32 *d_row = nullptr, *d_col = nullptr, *d_w = nullptr;
        TRYC(cudaMalloc((void**)&d_row, ((size_t)n + 1) * 4));
        TRYC(cudaMalloc((void**)&d_col, std::max<size_t>(1, (size_t)m) * 4));
        TRYC(cudaMalloc((void**)&d_w, std::max<size_t>(1, (size_t)m) * 4));
        const size_t bRow = ((size_t)n + 1) * 4, bCol = (size_t)m * 4, bW = (size_t)m * 4;
        char* stage = nullptr;
        cudaError_t e = cudaMallocHost((void**)&stage, 2 * bRow + bCol + bW);
        if (e != cudaSuccess) {
            cudaFree(d_row); cudaFree(d_col); cudaFree(d_w);
            cudaGetLastError();
            return bail(fail(PFG_ERR_OUT_OF_MEMORY, "pinned staging allocation failed"));
        }
        memcpy(stage, row, bRow);
        memcpy(stage + bRow, prow.data(), bRow);
        if (m) {
            memcpy(stage + 2 * bRow, col, bCol);
            memcpy(stage + 2 * bRow + bCol, w, bW);
        }
        cudaStream_t st[3];
        bool ok = true;
        for (auto& q : st) ok = ok && cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) == cudaSuccess;
        if (ok) {
            ok = cudaMemcpyAsync(d_row, stage, bRow, cudaMemcpyHostToDevice, st[0]) == cudaSuccess &&
                 cudaMemcpyAsync(s->d_prow, stage + bRow, bRow, cudaMemcpyHostToDevice, st[0]) == cudaSuccess &&
                 (m == 0 || cudaMemcpyAsync(d_col, stage + 2 * bRow, bCol, cudaMemcpyHostToDevice, st[1]) == cudaSuccess) &&
                 (m == 0 || cudaMemcpyAsync(d_w, stage + 2 * bRow + bCol, bW, cudaMemcpyHostToDevice, st[2]) == cudaSuccess);
            for (auto& q : st) {
                ok = cudaStreamSynchronize(q) == cudaSuccess && ok;
                cudaStreamDestroy(q);
            }
        }
        if (ok) ok = launch_build_adj(d_row, d_col, d_w, s->d_prow, n, s->d_adj, s->stream) == cudaSuccess;
        if (ok) ok = cudaStreamSynchronize(s->stream) == cudaSuccess;
        cudaFreeHost(stage);
        cudaFree(d_row);
        cudaFree(d_col);
        cudaFree(d_w);
        if (!ok) {
            cudaError_t le = cudaGetLastError();
            return bail(fail(PFG_ERR_CUDA, "CSR upload failed: %s", cudaGetErrorString(le)));
        }
    }
    if (s->has_xy) {
        TRY(s->dalloc(&s->d_x, n));
        TRY(s->dalloc(&s->d_y, n));
        // on the solver's stream: it does not wait for the legacy default stream
        TRYC(cudaMemcpyAsync(s->d_x, x, (size_t)n * 8, cudaMemcpyHostToDevice, s->stream));
        TRYC(cudaMemcpyAsync(s->d_y, y, (size_t)n * 8, cudaMemcpyHostToDevice, s->stream));
        TRYC(cudaStreamSynchronize(s->stream));
        s->hx.assign(x, x + n);
        s->hy.assign(y, y + n);
    }
    s->upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    // ---- working set, allocated once (reference: src/gpu_sssp.cu:160-186) ----
    TRY(s->dalloc(&s->d_state, Kn));
    for (int i = 0; i < 5; ++i) TRY(s->dalloc(&s->d_q[i], Kn));
    for (int i = 0; i < 3; ++i) {
        TRY(s->dalloc(&s->d_stamp[i], Kn));
        TRYC(cudaMemsetAsync(s->d_stamp[i], 0, Kn * 4, s->stream));
    }
    const u64 words = (u64)n / 32 + 1;
    for (int i = 0; i < 2; ++i) {
        TRY(s->dalloc(&s->d_naive[i], words));
        TRYC(cudaMemsetAsync(s->d_naive[i], 0, words * 4, s->stream));
    }
    // Ring of the asynchronous buckets: entries are queued per strict
    // improvement (several may be in flight for one vertex), so it has a power
    // of two >= 2 K n slots (at most 2^32: positions are u32 counters).
    u64 ring = 1024;
    while (ring < 2 * Kn && ring < (1ull << 32)) ring <<= 1;
    TRY(s->dalloc(&s->d_ring, ring));
    TRYC(cudaMemsetAsync(s->d_ring, 0xFF, ring * 8, s->stream));
    s->ring_mask = (u32)(ring - 1);
    TRY(s->dalloc(&s->d_aq, (u64)AQ_WORDS));
    TRYC(cudaMemsetAsync(s->d_aq, 0, AQ_WORDS * 4, s->stream));
    // Independent bucket windows: per-instance windows, pending counts and far-pile
    // counters (every run that uses them rewrites the block first).
    // Sized for runs of up to IW_MAX_INST sources whatever maxBatch is (each run checks its own k).
    {
        const u32 kw = std::min<u32>(K, IW_MAX_INST);
        if ((u64)kw * n < (u64)IW_FAR_BIT) TRY(s->dalloc(&s->d_iw, iw_words(kw)));
    }
    // Hub records: every instance's hub rows once per round, twice over for
    // re-published rows of an asynchronous drain (overflow falls back to the CTA).
    if (s->hub_rows) {
        s->hub_cap = (u32)std::min<u64>(std::max<u64>(1024, 2 * (u64)K * s->hub_rows), 1u << 24);
        TRY(s->dalloc(&s->d_hubs, (u64)s->hub_cap));
        TRYC(cudaMemsetAsync(s->d_hubs, 0, (size_t)s->hub_cap * sizeof(HubRec), s->stream));
    }
    TRY(s->dalloc(&s->d_srcs, K));
    TRY(s->dalloc(&s->d_path, (u64)n + 1));
    TRY(s->dalloc(&s->d_path_len, 1));
    TRY(s->dalloc(&s->d_ctl, 1));
    TRY(s->dalloc(&s->d_net, 1));
    TRYC(cudaMallocHost((void**)&s->h_ctl, sizeof(Ctl)));
    TRYC(cudaMallocHost((void**)&s->h_srcs, (size_t)K * 4));
    memset(s->h_ctl, 0, sizeof(Ctl));
    s->h_ctl->near_epoch = 1;
    s->h_ctl->far_epoch = 1;
    s->h_ctl->r_epoch = 1;
    TRYC(cudaMemcpyAsync(s->d_ctl, s->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, s->stream));
    TRYC(cudaStreamSynchronize(s->stream));
    *out = s;
    return PFG_OK;
#undef TRY
#undef TRYC
}

extern "C" pfg_status pfg_create(const uint32_t* row, const uint32_t* col, const uint32_t* w,
                                 const double* x, const double* y, uint32_t n, uint32_t m,
                                 double h_scale, double avg_w, double avg_deg, uint32_t max_batch,
                                 pfg_solver** out) {
    return pfg_create_on_device(row, col, w, x, y, n, m, h_scale, avg_w, avg_deg, max_batch, 0, out);
}

extern "C" void pfg_destroy(pfg_solver* s) { destroy_solver(s); }
extern "C" double pfg_upload_ms(const pfg_solver* s) { return s ? s->upload_ms : 0.0; }
extern "C" uint64_t pfg_device_bytes(const pfg_solver* s) { return s ? s->bytes : 0; }
extern "C" uint32_t pfg_auto_delta(const pfg_solver* s) {
    return s ? auto_delta_of(s->avg_w, s->avg_deg) : 0u;
}
extern "C" uint32_t pfg_num_vertices(const pfg_solver* s) { return s ? s->n : 0u; }
extern "C" uint32_t pfg_max_batch(const pfg_solver* s) { return s ? s->K : 0u; }
extern "C" void* pfg_stream(const pfg_solver* s) { return s ? (void*)s->stream : nullptr; }
extern "C" const uint64_t* pfg_state_device(const pfg_solver* s) { return s ? s->d_state : nullptr; }

// ---------------------------------------------------------------------------
// Runs
// ---------------------------------------------------------------------------
static int env_int(const char* name, int dflt) {
    const char* v = getenv(name);
    if (!v || !*v) return dflt;
    return atoi(v);
}

namespace pfg {

pfg_options default_options() {
    pfg_options o;
    o.algo = PFG_ALGO_DELTA;
    o.mapping = PFG_MAP_HYBRID;
    o.atomic = PFG_ATOMIC_MIN_RBA;
    o.delta = 0;
    o.block_size = 256;
    o.sync_every = 8;
    o.compaction = PFG_COMPACT_WARP_ATOMIC;
    o.policy = PFG_POLICY_FIXED;
    o.eager = -1;
    o.blocks_per_sm = 0;
    o.schedule = PFG_SCHEDULE_AUTO;
    return o;
}

void sanitize_options(pfg_options& o) {
    // Silent fix-up of the reference (src/gpu_sssp.cu:462).
    if (o.block_size < 32 || o.block_size > 1024 || (o.block_size % 32) != 0) o.block_size = 256;
    if (o.mapping < 0 || o.mapping > 2) o.mapping = PFG_MAP_HYBRID;
    if (o.atomic < 0 || o.atomic > 2) o.atomic = PFG_ATOMIC_MIN_RBA;
    if (o.schedule < 0 || o.schedule > 4) o.schedule = PFG_SCHEDULE_AUTO;
}

int blocks_per_sm_for(const pfg_options& o, bool astar, int map, bool iw, u32 k) {
    int bps = persistent_blocks_per_sm(astar, o.atomic, map, o.block_size, false, iw ? k : 0u);
    if (bps <= 0) return 0;
    // Default: fill each SM up to 1024 resident threads (more CTAs only make
    // the grid barrier slower on this latency-bound kernel).
    int want = o.blocks_per_sm > 0 ? o.blocks_per_sm : std::max(1, 1024 / o.block_size);
    const int cap = env_int("PFG_BLOCKS_PER_SM", 0);
    if (cap > 0) want = cap;
    return std::max(1, std::min(bps, want));
}

u32 eager_rounds_for(const pfg_options& o) {
    return o.eager < 0 ? (u32)std::max(0, env_int("PFG_EAGER", kDefaultEager)) : (u32)o.eager;
}

u64 device_timeout_ns() { return (u64)std::max(1, env_int("PFG_TIMEOUT_MS", 2000)) * 1000000ull; }

void configure_drain(RunParams& p, int schedule, HubRec* hubs, u32 hub_cap, u32 max_deg, u32* aq, int mapping,
                     int block) {
    p.warp_drain = (p.ring && mapping == PFG_MAP_HYBRID && schedule == PFG_SCHEDULE_WARP) ? 1u : 0u;
    // Rows of more than 256 selected arcs are worked by every warp of the CTA
    // (row tasks); rows beyond the CTA tier (hub_min) also by other CTAs, which
    // claim 256 arcs of them at a time.
    p.hub_min_warp = (u32)std::max(32, env_int("PFG_HUB_WARP", 256));
    p.hub_chunk_warp = 256u;
    // Block-synchronous drain: on graphs of short rows a CTA keeps up to half its
    // claimed list before it spills while no CTA is idle (large batches: 12-13 %
    // faster at 128-256 instances on the 1000 x 1000 grid); elsewhere half a block
    // (hub rows make spilled work pay off sooner).
    p.spill_keep = (u32)std::max(0, env_int("PFG_SPILL_KEEP", p.short_rows ? 1024 : 0));
    p.idle_ns = (u32)std::max(0, env_int("PFG_IDLE_NS", 64));
    if (p.ring && p.warp_drain && hubs && mapping == PFG_MAP_HYBRID && max_deg > 8u * (u32)block && !p.hubs) {
        p.hubs = hubs;
        p.hub_cap = hub_cap;
        p.hub_min = 8u * (u32)block;
        p.hub_chunk = 4u * (u32)block;
        p.aq = aq;
    }
}

bool async_buckets_for(const pfg_options& o, int mode) {
    // Delta-stepping only: Frontier relaxation drained as one unbounded
    // asynchronous bucket relaxes 4-6x the arcs of its eager rounds on road grids
    return o.schedule != PFG_SCHEDULE_ROUNDS && mode == MODE_DELTA;
}

}  // namespace pfg

// Resets the stamp words when the epoch counters approach 2^32 (2^31 for a run
// under independent windows, whose far epochs share a word with a pile index).
static pfg_status maybe_reset_epochs(pfg_solver* s, bool iw) {
    if (s->epoch_hint < (iw ? 0x70000000u : 0xF0000000u)) return PFG_OK;
    const u64 Kn = (u64)s->K * s->n;
    for (int i = 0; i < 3; ++i) PFG_CUDA(cudaMemsetAsync(s->d_stamp[i], 0, Kn * 4, s->stream));
    Ctl tmp;
    memset(&tmp, 0, sizeof(tmp));
    tmp.near_epoch = tmp.far_epoch = tmp.r_epoch = 1;
    const size_t off = offsetof(Ctl, persist);
    PFG_CUDA(cudaMemcpyAsync((char*)s->d_ctl + off, (char*)&tmp + off, sizeof(Ctl) - off,
                             cudaMemcpyHostToDevice, s->stream));
    PFG_CUDA(cudaStreamSynchronize(s->stream));
    s->epoch_hint = 1;
    return PFG_OK;
}

// Enqueues one run on the solver's stream. h_srcs (host) or d_srcs (device).
static pfg_status enqueue_run(pfg_solver* s, const uint32_t* h_srcs, const uint32_t* d_srcs,
                              uint32_t k, int32_t astar, uint32_t dst, const pfg_options* opt_in,
                              bool timed, float* d_trace = nullptr, u32 trace_cap = 0) {
    if (!s) return fail(PFG_ERR_INVALID_ARGUMENT, "solver is NULL");
    pfg_options o = opt_in ? *opt_in : default_options();
    sanitize_options(o);
    if (k == 0 || k > s->K) return fail(PFG_ERR_INVALID_ARGUMENT, "invalid batch size");
    if (h_srcs) {
        for (u32 i = 0; i < k; ++i)
            if (h_srcs[i] >= s->n) return fail(PFG_ERR_INVALID_ARGUMENT, "source out of range");
    } else if (!d_srcs) {
        return fail(PFG_ERR_INVALID_ARGUMENT, "sources are NULL");
    }
    if (astar && dst >= s->n) return fail(PFG_ERR_INVALID_ARGUMENT, "target out of range");
    if (astar && k != 1) return fail(PFG_ERR_INVALID_ARGUMENT, "A* runs take exactly one source");
    if (o.algo < 0 || o.algo > 2) return fail(PFG_ERR_INVALID_ARGUMENT, "unknown algorithm %d", o.algo);
    if (o.algo == PFG_ALGO_NAIVE && k > 1) o.algo = PFG_ALGO_DELTA;
    if (o.policy == PFG_POLICY_LEARNED && !s->has_net)
        return fail(PFG_ERR_INVALID_ARGUMENT, "learned policy requested but no network is loaded");
    PFG_CUDA(cudaSetDevice(s->device));

    const int mode = o.algo == PFG_ALGO_NAIVE ? MODE_NAIVE
                   : o.algo == PFG_ALGO_FRONTIER ? MODE_FRONTIER : MODE_DELTA;
    u32 delta = mode == MODE_DELTA ? (o.delta ? o.delta : auto_delta_of(s->avg_w, s->avg_deg)) : 0u;
    // Independent bucket windows: multi-source Delta-stepping with the hybrid mapping's
    // CTA passes, every arc light (Delta >= the largest weight), no hub rows and no
    // learned policy or trace. Each instance's run is then bound by its own buckets, one
    // after the other, so the automatic Delta is widened (4x, PFG_IW_DELTA_MULT): the
    // extra relaxations of wider windows overlap with other instances' work (1000 x 1000
    // grid, 256 sources: 56.9 ms with a shared window at the automatic Delta, 35.9 ms).
    // The automatic schedule takes them from 96 instances on (PFG_INST_WINDOWS: the
    // smallest batch, 0 = never), where they measured faster; PFG_SCHEDULE_INSTANCE asks
    // for them at any batch size and falls back to a shared window where they do not apply.
    const u64 iw_delta = o.delta ? (u64)o.delta
                                 : (u64)delta * (u64)std::max(1, env_int("PFG_IW_DELTA_MULT", 4));
    const bool iw_fits = mode == MODE_DELTA && !astar && k > 1 && s->d_iw && k <= IW_MAX_INST &&
                         (u64)k * s->n < (u64)IW_FAR_BIT && iw_delta >= s->maxw && iw_delta < 0x80000000ull &&
                         o.mapping == PFG_MAP_HYBRID && o.policy != PFG_POLICY_LEARNED && !d_trace &&
                         s->max_deg <= 8u * (u32)o.block_size &&
                         o.block_size >= 64;  // (warp 0 of a CTA serves, the others relax)
    const int iw_min = env_int("PFG_INST_WINDOWS", 96);
    const bool iw = iw_fits && (o.schedule == PFG_SCHEDULE_INSTANCE ||
                                (o.schedule == PFG_SCHEDULE_AUTO && iw_min > 0 && (int)k >= iw_min));
    if (iw) delta = (u32)iw_delta;
    pfg_status st = maybe_reset_epochs(s, iw);
    if (st != PFG_OK) return st;

    // Control block for this run (the persistent epoch part is left alone).
    Ctl* c = s->h_ctl;
    const size_t run_bytes = offsetof(Ctl, persist);
    memset(c, 0, run_bytes);
    c->rd.phase = PH_INIT;
    c->rd.far_out = 0;
    c->rd.map_mode = 1u;
    c->far_min[0] = c->far_min[1] = ~0ull;
    const u64 cap = 4ull * s->n + 1000ull;
    c->round_cap = (u32)std::min<u64>(cap, 0x7FFFFFFFull);
    c->rd.delta = delta ? delta : 1u;
    c->delta0 = delta;
    c->rd.heavy = (mode == MODE_DELTA && delta < s->maxw) ? 1u : 0u;

    RunParams p;
    memset(&p, 0, sizeof(p));
    p.adj = s->d_adj;
    p.prow = s->d_prow;
    p.row_stride = s->row_stride;
    p.short_rows = s->max_deg <= 32u ? 1u : 0u;
    p.x = s->d_x;
    p.y = s->d_y;
    p.n = s->n;
    p.maxw = s->maxw;
    p.hscale = s->hscale;
    p.avg_w = s->avg_w;
    p.avg_deg = s->avg_deg;
    p.m = s->m;
    p.k = k;
    p.total = k * s->n;
    p.srcs = d_srcs ? d_srcs : s->d_srcs;
    p.astar = astar ? 1 : 0;
    p.target = astar ? dst : 0u;
    p.use_h = (astar && s->has_xy && s->hscale > 0.0) ? 1 : 0;
    if (p.use_h) {
        p.xt = s->hx[dst];
        p.yt = s->hy[dst];
    }
    p.state = s->d_state;
    p.nearq[0] = s->d_q[0];
    p.nearq[1] = s->d_q[1];
    p.farq[0] = s->d_q[2];
    p.farq[1] = s->d_q[3];
    p.rq = s->d_q[4];
    p.near_stamp = s->d_stamp[0];
    p.far_stamp = s->d_stamp[1];
    p.r_stamp = s->d_stamp[2];
    p.naive_mask[0] = s->d_naive[0];
    p.naive_mask[1] = s->d_naive[1];
    p.ctl = s->d_ctl;
    p.delta = delta ? delta : 1u;
    p.mode = mode;
    p.prefix_scan = (mode == MODE_FRONTIER && o.compaction == PFG_COMPACT_PREFIX_SCAN) ? 1 : 0;
    p.policy = (mode == MODE_DELTA && o.policy == PFG_POLICY_LEARNED) ? 1 : 0;
    p.eager = eager_rounds_for(o);
    // Engine default: eager propagation only on low-degree (road-like) graphs;
    // on power-law graphs one hub expands into a burst of redundant work.
    if (o.eager < 0 && s->avg_deg > kEagerMaxAvgDegree) p.eager = 0;
    p.net = s->d_net;
    p.trace = mode == MODE_DELTA ? d_trace : nullptr;
    p.trace_cap = trace_cap;
    p.timeout_ns = device_timeout_ns();
    p.test_absent_cta = env_int("PFG_TEST_ABSENT_CTA", 0) != 0 ? 1 : 0;
    // Asynchronous buckets for Delta-stepping (see pfg_schedule).
    if (async_buckets_for(o, mode)) {
        p.ring = s->d_ring;
        p.ring_mask = s->ring_mask;
        p.aq = s->d_aq;
    }

    // The naive sweep deals each mask word's arcs over a warp whatever the
    // mapping; its thread-mapping instantiation measured fastest.
    const int map = mode == MODE_NAIVE ? PFG_MAP_THREAD : o.mapping;
    const int block = o.block_size;
    // Grid tier of the hybrid mapping for rows longer than 8 CTAs' worth of arcs, claimed
    // in chunks of 4 CTAs' worth. A single source with 1024-thread CTAs publishes rows
    // above 4,096 arcs and claims 2,048 at a time (R-MAT-20: ~10 % faster; with 16
    // sources the larger tier wins). PFG_HUB_BLOCKS / PFG_HUB_CHUNK_BLOCKS override both,
    // in blocks.
    u32 hub_min = 8u * (u32)block, hub_chunk = 4u * (u32)block;
    if (k == 1) {
        hub_min = std::min(hub_min, 4096u);
        hub_chunk = std::min(hub_chunk, 2048u);
    }
    if (env_int("PFG_HUB_BLOCKS", 0) > 0) hub_min = (u32)env_int("PFG_HUB_BLOCKS", 0) * (u32)block;
    if (env_int("PFG_HUB_CHUNK_BLOCKS", 0) > 0) hub_chunk = (u32)env_int("PFG_HUB_CHUNK_BLOCKS", 0) * (u32)block;
    hub_min = std::max(hub_min, 256u);  // the records are sized for rows above 256 arcs
    if (s->d_hubs && (map == PFG_MAP_HYBRID || mode == MODE_NAIVE) && s->max_deg > hub_min) {
        p.hubs = s->d_hubs;
        p.hub_cap = s->hub_cap;
        p.hub_min = hub_min;
        p.hub_chunk = hub_chunk;
        p.aq = s->d_aq;
    }
    configure_drain(p, o.schedule, s->d_hubs, s->hub_cap, s->max_deg, s->d_aq, map, block);
    if (iw) {
        p.iw = 1u;
        p.iw_win = reinterpret_cast<unsigned long long*>(s->d_iw);
        p.iw_pend = s->d_iw + 2u * k;
        p.iw_fcnt = s->d_iw + 3u * k;
        p.iw_fmin = s->d_iw + 5u * k;
        p.iw_misc = s->d_iw + 7u * k;
        p.hubs = nullptr;  // (no row reaches the grid tier: max_deg <= 8 blocks)
    }
    // A single source on a graph of short rows is bound by the latency of its hops: its
    // entries are relaxed without the state read (1000 x 1000 grid: 6.22 -> 5.79 ms); with
    // more instances the stale entries' extra work costs more than it saves (K = 64:
    // 14.6 -> 18.3 ms), so they keep the check.
    p.trust_entries = (k == 1 && p.short_rows && env_int("PFG_TRUST_ENTRIES", 1) != 0) ? 1u : 0u;
    const int bps = blocks_per_sm_for(o, astar != 0, map, iw, k);
    if (bps <= 0) return fail(PFG_ERR_CUDA, "occupancy query failed for block size %d", block);
    const int grid = s->sm_count * bps;
    // Eager propagation pays in rounds that leave most of the GPU idle: inputs
    // of at most a quarter of the launched threads.
    p.eager_max_items = (u32)std::max<long long>(1, (long long)grid * block / 4);

    if (timed) PFG_CUDA(cudaEventRecord(s->ev0, s->stream));
    if (h_srcs) {
        memcpy(s->h_srcs, h_srcs, (size_t)k * 4);
        PFG_CUDA(cudaMemcpyAsync(s->d_srcs, s->h_srcs, (size_t)k * 4, cudaMemcpyHostToDevice, s->stream));
    }
    PFG_CUDA(cudaMemcpyAsync(s->d_ctl, c, run_bytes, cudaMemcpyHostToDevice, s->stream));
    cudaError_t le = launch_persistent(p, astar != 0, o.atomic, map, block, grid, s->stream);
    if (le != cudaSuccess) {
        cudaGetLastError();
        return fail(PFG_ERR_CUDA, "persistent launch failed (grid %d x %d): %s", grid, block,
                    cudaGetErrorString(le));
    }
    if (timed) PFG_CUDA(cudaEventRecord(s->ev1, s->stream));
    PFG_CUDA(cudaMemcpyAsync(c, s->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
    s->pending = true;
    s->last_mode = mode;
    s->last_delta = delta;
    s->last_k = k;
    s->last_iw = iw;
    return PFG_OK;
}

// Waits for the enqueued run and converts its control block into stats/status.
static pfg_status complete_run(pfg_solver* s, pfg_stats* stats_out) {
    if (!s->pending) return fail(PFG_ERR_INVALID_ARGUMENT, "no run in flight");
    s->pending = false;
    PFG_CUDA(cudaStreamSynchronize(s->stream));
    const Ctl* c = s->h_ctl;
    s->epoch_hint = std::max({c->near_epoch, c->far_epoch, c->r_epoch});
    // Independent windows advance the far epochs inside the drain and record the last one at
    // the final transition; a run that failed before it may have left newer stamps, so the
    // stamp words are cleared before the next run.
    if (s->last_iw && c->rd.status != DS_OK) s->epoch_hint = 0xFFFFFFFFu;
    if (stats_out) {
        memset(stats_out, 0, sizeof(*stats_out));
        stats_out->edges_scanned = c->stats[0];
        stats_out->atomics_issued = c->stats[1];
        stats_out->updates = c->stats[2];
        stats_out->pushes = c->stats[3];
        stats_out->iterations = c->iterations;
        stats_out->host_syncs = 1;
        stats_out->launches = 1;
        stats_out->buckets = s->last_mode == MODE_DELTA ? c->buckets : 0u;
        stats_out->delta = s->last_delta;
        stats_out->rounds = c->rounds;
    }
    const u32 status = c->rd.status;
    if (status != DS_OK && status != DS_TIMEOUT) {
        // (a run that ended early may leave ring entries behind)
        cudaMemsetAsync(s->d_ring, 0xFF, ((u64)s->ring_mask + 1) * 8, s->stream);
        cudaMemsetAsync(s->d_aq, 0, AQ_WORDS * 4, s->stream);
    }
    if (status == DS_TIMEOUT) {
        // A wait gave up: reset the naive masks and the ring so the next run starts clean.
        const u64 words = (u64)s->n / 32 + 1;
        for (int i = 0; i < 2; ++i) cudaMemsetAsync(s->d_naive[i], 0, words * 4, s->stream);
        cudaMemsetAsync(s->d_ring, 0xFF, ((u64)s->ring_mask + 1) * 8, s->stream);
        cudaMemsetAsync(s->d_aq, 0, AQ_WORDS * 4, s->stream);
        cudaStreamSynchronize(s->stream);
        return fail(PFG_ERR_DEVICE_TIMEOUT, "device-side wait timed out: %s made no progress for %llu ms",
                    wait_site_name(c->wait_site), (unsigned long long)(device_timeout_ns() / 1000000ull));
    }
    if (status == DS_NOT_CONVERGED) {
        const u64 words = (u64)s->n / 32 + 1;
        for (int i = 0; i < 2; ++i) cudaMemsetAsync(s->d_naive[i], 0, words * 4, s->stream);
        cudaStreamSynchronize(s->stream);
        const char* what = s->last_mode == MODE_NAIVE ? "Naive relaxation"
                         : s->last_mode == MODE_FRONTIER ? "Frontier relaxation" : "Delta-stepping";
        return fail(PFG_ERR_NOT_CONVERGED, "%s did not converge", what);
    }
    if (status == DS_BAD_SOURCE) return fail(PFG_ERR_INVALID_ARGUMENT, "source out of range");
    if (status != DS_OK) return fail(PFG_ERR_CUDA, "device status %u", status);
    return PFG_OK;
}

// ---------------------------------------------------------------------------
// Streamed multi-source runs
// ---------------------------------------------------------------------------
// Splits the finished streamed run's distances into d_dist (once the previous
// copy has drained it) and starts their copy to pipe_out on the copy stream.
// The run's kernel has completed (complete_run).
static pfg_status pipe_start_copy(pfg_solver* s) {
    if (!s->pipe_out) return PFG_OK;
    const u64 count = (u64)s->pipe_k * s->n;
    uint32_t* out = s->pipe_out;
    s->pipe_out = nullptr;
    PFG_CUDA(cudaStreamWaitEvent(s->stream, s->ev_copied, 0));
    const cudaError_t e = launch_extract_dist(s->d_state, count, s->d_dist, s->sm_count, s->stream);
    if (e != cudaSuccess) return fail(PFG_ERR_CUDA, "distance extraction: %s", cudaGetErrorString(e));
    PFG_CUDA(cudaEventRecord(s->ev_split, s->stream));
    PFG_CUDA(cudaStreamWaitEvent(s->copy_stream, s->ev_split, 0));
    PFG_CUDA(cudaMemcpyAsync(out, s->d_dist, count * 4, cudaMemcpyDeviceToHost, s->copy_stream));
    PFG_CUDA(cudaEventRecord(s->ev_copied, s->copy_stream));
    s->pipe_copying = true;
    return PFG_OK;
}

// Completes a stream of runs: the last run's kernel, its split and copy, and
// every copy still in flight.
static pfg_status pipe_flush(pfg_solver* s, pfg_stats* stats_out) {
    PFG_CUDA(cudaSetDevice(s->device));
    pfg_status st = PFG_OK;
    if (s->pipe_out) {
        st = complete_run(s, stats_out);
        if (st == PFG_OK) st = pipe_start_copy(s);
        s->pipe_out = nullptr;
    }
    if (s->pipe_copying) {
        const cudaError_t e = cudaStreamSynchronize(s->copy_stream);
        s->pipe_copying = false;
        if (e != cudaSuccess && st == PFG_OK)
            st = fail(PFG_ERR_CUDA, "distance copy failed: %s", cudaGetErrorString(e));
    }
    return st;
}

// Every other entry point first completes a stream of runs in flight.
#define PIPE_FLUSH(s)                                          \
    do {                                                       \
        if ((s)->pipe_out || (s)->pipe_copying) {              \
            const pfg_status pst__ = pipe_flush((s), nullptr); \
            if (pst__ != PFG_OK) return pst__;                 \
        }                                                      \
    } while (0)

extern "C" pfg_status pfg_run_dist_async(pfg_solver* s, const uint32_t* h_srcs, uint32_t k,
                                         const pfg_options* opt, uint32_t* h_dist_out,
                                         pfg_stats* prev_stats_out) {
    if (!s) return fail(PFG_ERR_INVALID_ARGUMENT, "solver is NULL");
    if (!h_srcs || !h_dist_out) return fail(PFG_ERR_INVALID_ARGUMENT, "sources or output are NULL");
    PFG_CUDA(cudaSetDevice(s->device));
    if (!s->copy_stream) {
        PFG_CUDA(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        PFG_CUDA(cudaEventCreateWithFlags(&s->ev_split, cudaEventDisableTiming));
        PFG_CUDA(cudaEventCreateWithFlags(&s->ev_copied, cudaEventDisableTiming));
    }
    if (!s->d_dist) {
        const pfg_status st = s->dalloc(&s->d_dist, (u64)s->K * s->n);
        if (st != PFG_OK) return st;
    }
    if (s->pipe_out) {
        // the previous streamed run: wait for its kernel, then copy its distances
        // while the run enqueued below computes
        pfg_status st = complete_run(s, prev_stats_out);
        if (st != PFG_OK) {
            s->pipe_out = nullptr;
            return st;
        }
        st = pipe_start_copy(s);
        if (st != PFG_OK) return st;
    } else if (s->pending) {
        const pfg_status st = complete_run(s, nullptr);
        (void)st;
    }
    const pfg_status st = enqueue_run(s, h_srcs, nullptr, k, 0, 0, opt, true);
    if (st != PFG_OK) return st;
    s->pipe_out = h_dist_out;
    s->pipe_k = k;
    return PFG_OK;
}

extern "C" pfg_status pfg_dist_wait(pfg_solver* s, pfg_stats* stats_out) {
    if (!s) return fail(PFG_ERR_INVALID_ARGUMENT, "solver is NULL");
    PFG_CUDA(cudaSetDevice(s->device));
    return pipe_flush(s, stats_out);
}

extern "C" pfg_status pfg_run(pfg_solver* s, const uint32_t* h_srcs, uint32_t k, int32_t astar,
                              uint32_t dst, const pfg_options* opt, pfg_stats* stats_out,
                              uint64_t* h_state_out, float* ms_out) {
    if (!s) return fail(PFG_ERR_INVALID_ARGUMENT, "solver is NULL");
    if (!h_srcs) return fail(PFG_ERR_INVALID_ARGUMENT, "sources are NULL");
    PIPE_FLUSH(s);
    if (s->pending) {
        pfg_status st = complete_run(s, nullptr);
        (void)st;
    }
    pfg_status st = enqueue_run(s, h_srcs, nullptr, k, astar, dst, opt, true);
    if (st != PFG_OK) return st;
    st = complete_run(s, stats_out);
    if (st != PFG_OK) return st;
    if (ms_out) {
        float ms = 0.f;
        PFG_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
        *ms_out = ms;
    }
    if (h_state_out) {
        PFG_CUDA(cudaMemcpyAsync(h_state_out, s->d_state, (size_t)k * s->n * 8,
                                 cudaMemcpyDeviceToHost, s->stream));
        PFG_CUDA(cudaStreamSynchronize(s->stream));
    }
    return PFG_OK;
}

extern "C" pfg_status pfg_run_traced(pfg_solver* s, const uint32_t* h_srcs, uint32_t k,
                                     const pfg_options* opt, pfg_stats* stats_out, float* h_trace,
                                     uint32_t trace_cap, uint32_t* rows_out, float* ms_out) {
    if (!s || !h_srcs || !h_trace || !rows_out || trace_cap == 0)
        return fail(PFG_ERR_INVALID_ARGUMENT, "pfg_run_traced: bad argument");
    PIPE_FLUSH(s);
    PFG_CUDA(cudaSetDevice(s->device));
    if (s->pending) complete_run(s, nullptr);
    if (trace_cap > s->trace_cap) {
        if (s->d_trace) cudaFree(s->d_trace);
        s->d_trace = nullptr;
        s->trace_cap = 0;
        PFG_CUDA(cudaMalloc((void**)&s->d_trace, (size_t)trace_cap * TRACE_W * sizeof(float)));
        s->trace_cap = trace_cap;
    }
    pfg_status st = enqueue_run(s, h_srcs, nullptr, k, 0, 0, opt, true, s->d_trace, trace_cap);
    if (st != PFG_OK) return st;
    st = complete_run(s, stats_out);
    if (st != PFG_OK) return st;
    if (ms_out) PFG_CUDA(cudaEventElapsedTime(ms_out, s->ev0, s->ev1));
    const u32 rows = std::min(s->h_ctl->buckets, trace_cap);
    *rows_out = rows;
    if (rows) PFG_CUDA(cudaMemcpy(h_trace, s->d_trace, (size_t)rows * TRACE_W * sizeof(float), cudaMemcpyDeviceToHost));
    return PFG_OK;
}

extern "C" pfg_status pfg_run_async(pfg_solver* s, const uint32_t* d_srcs, uint32_t k,
                                    int32_t astar, uint32_t dst, const pfg_options* opt) {
    if (!s) return fail(PFG_ERR_INVALID_ARGUMENT, "solver is NULL");
    if (!d_srcs) return fail(PFG_ERR_INVALID_ARGUMENT, "sources are NULL");
    PIPE_FLUSH(s);
    if (s->pending) {
        pfg_status st = complete_run(s, nullptr);
        (void)st;
    }
    return enqueue_run(s, nullptr, d_srcs, k, astar, dst, opt, false);
}

extern "C" pfg_status pfg_finish(pfg_solver* s, pfg_stats* stats_out) {
    if (!s) return fail(PFG_ERR_INVALID_ARGUMENT, "solver is NULL");
    PIPE_FLUSH(s);
    return complete_run(s, stats_out);
}

extern "C" pfg_status pfg_copy_state(pfg_solver* s, uint64_t first, uint64_t count, uint64_t* h_out) {
    if (!s || !h_out) return fail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    PIPE_FLUSH(s);
    // (written so that no sum can wrap around 2^64)
    const u64 total_states = (u64)s->K * s->n;
    if (first > total_states || count > total_states - first)
        return fail(PFG_ERR_INVALID_ARGUMENT, "range outside the state");
    PFG_CUDA(cudaSetDevice(s->device));
    if (s->pending) {
        pfg_status st = complete_run(s, nullptr);
        if (st != PFG_OK) return st;
    }
    PFG_CUDA(cudaMemcpyAsync(h_out, s->d_state + first, count * 8, cudaMemcpyDeviceToHost, s->stream));
    PFG_CUDA(cudaStreamSynchronize(s->stream));
    return PFG_OK;
}

extern "C" pfg_status pfg_copy_dist(pfg_solver* s, uint64_t first, uint64_t count, uint32_t* h_out) {
    if (!s || (count > 0 && !h_out)) return fail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    PIPE_FLUSH(s);
    // (written so that no sum can wrap around 2^64)
    const u64 total_states = (u64)s->K * s->n;
    if (first > total_states || count > total_states - first)
        return fail(PFG_ERR_INVALID_ARGUMENT, "range outside the state");
    PFG_CUDA(cudaSetDevice(s->device));
    if (s->pending) {
        pfg_status st = complete_run(s, nullptr);
        if (st != PFG_OK) return st;
    }
    if (count == 0) return PFG_OK;
    // near queue 0 (K*n words) is free scratch between runs
    cudaError_t e = launch_extract_dist(s->d_state + first, count, s->d_q[0], s->sm_count, s->stream);
    if (e != cudaSuccess) return fail(PFG_ERR_CUDA, "distance extraction: %s", cudaGetErrorString(e));
    PFG_CUDA(cudaMemcpyAsync(h_out, s->d_q[0], count * 4, cudaMemcpyDeviceToHost, s->stream));
    PFG_CUDA(cudaStreamSynchronize(s->stream));
    return PFG_OK;
}

extern "C" pfg_status pfg_extract_path(pfg_solver* s, uint32_t inst, uint32_t src, uint32_t dst,
                                       uint32_t* h_path, uint32_t cap, uint32_t* path_len_out) {
    if (!s || !path_len_out || (cap > 0 && !h_path)) return fail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (inst >= s->K || src >= s->n || dst >= s->n)
        return fail(PFG_ERR_INVALID_ARGUMENT, "instance, source or target out of range");
    PIPE_FLUSH(s);
    PFG_CUDA(cudaSetDevice(s->device));
    if (s->pending) {
        pfg_status st = complete_run(s, nullptr);
        if (st != PFG_OK) return st;
    }
    const u32 dcap = std::min<u32>(cap, s->n + 1);
    cudaError_t e = launch_extract_path(s->d_state, (u64)inst * s->n, s->n, src, dst, s->d_path,
                                        s->n + 1, s->d_path_len, s->stream);
    if (e != cudaSuccess) return fail(PFG_ERR_CUDA, "path kernel: %s", cudaGetErrorString(e));
    u32 len = 0;
    PFG_CUDA(cudaMemcpyAsync(&len, s->d_path_len, 4, cudaMemcpyDeviceToHost, s->stream));
    PFG_CUDA(cudaStreamSynchronize(s->stream));
    *path_len_out = 0;
    if (len == 0) return PFG_OK;
    if (len > dcap) {
        *path_len_out = len;
        return fail(PFG_ERR_CAPACITY, "path has %u vertices, buffer holds %u", len, cap);
    }
    std::vector<u32> rev(len);
    PFG_CUDA(cudaMemcpy(rev.data(), s->d_path, (size_t)len * 4, cudaMemcpyDeviceToHost));
    for (u32 i = 0; i < len; ++i) h_path[i] = rev[len - 1 - i];
    *path_len_out = len;
    return PFG_OK;
}

// Loads a learned-policy network (host PolicyNet image) into the solver.
extern "C" pfg_status pfg_set_policy(pfg_solver* s, const float* params, uint64_t count) {
    if (!s || !params) return fail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    PIPE_FLUSH(s);
    if (count * sizeof(float) != sizeof(PolicyNet))
        return fail(PFG_ERR_INVALID_ARGUMENT, "policy image has %llu floats, expected %llu",
                    (unsigned long long)count, (unsigned long long)(sizeof(PolicyNet) / sizeof(float)));
    PFG_CUDA(cudaSetDevice(s->device));
    if (s->pending) {
        pfg_status st = complete_run(s, nullptr);
        if (st != PFG_OK) return st;
    }
    PFG_CUDA(cudaMemcpyAsync(s->d_net, params, sizeof(PolicyNet), cudaMemcpyHostToDevice, s->stream));
    PFG_CUDA(cudaStreamSynchronize(s->stream));
    s->has_net = true;
    return PFG_OK;
}

extern "C" uint64_t pfg_policy_param_count(void) { return sizeof(PolicyNet) / sizeof(float); }
