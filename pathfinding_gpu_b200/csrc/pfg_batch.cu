// pfg_batch.cu - many graphs of uneven sizes and many sources in one launch.
//
// The reference batches K sources of ONE graph with state index k*n + v
// (src/gpu_kernels.cuh:223-225, src/gpu_sssp.cu:553-569). A batch here holds
// several graphs (their padded adjacencies concatenated in one array) and a
// table of instances (graph, source); instance i owns the state words
// [inst_off[i], inst_off[i+1]) and its graph's rows start at
// prow[inst_rowbase[i]]. One persistent launch relaxes every instance, with a
// shared bucket sequence, exactly like the uniform multi-source run. A run can
// be recorded once into a CUDA graph and replayed, which removes the host-side
// launch work of repeated batches.
#include "../../include/pfg.h"
#include "pfg_common.cuh"
#include "pfg_internal.h"
#include "pfg_kernels.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

using namespace pfg;

struct pfg_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int sm_count = 1;
    u32 num_graphs = 0;
    std::vector<u32> g_n, g_m, g_rowbase;
    u32 maxw = 0;
    u32 max_deg = 0;
    u32 row_stride = 0;  // ROW_ALIGN when every row of every graph has exactly ROW_ALIGN slots
    u64 hub_rows = 0;  // vertices with more than 256 arcs (all graphs)
    double avg_w = 0.0, avg_deg = 0.0;
    u64 max_states = 0;
    u32 max_inst = 0;
    u32 num_inst = 0;
    u64 total_states = 0;
    std::vector<u32> inst_off;
    double upload_ms = 0.0;
    u64 bytes = 0;

    uint2* d_adj = nullptr;
    u32* d_prow = nullptr;
    u64* d_state = nullptr;
    u32* d_q[5] = {};
    u32* d_stamp[3] = {};
    u32* d_inst_off = nullptr;
    u32* d_inst_rowbase = nullptr;
    u32* d_srcs = nullptr;
    unsigned long long* d_ring = nullptr;  // ring queue of asynchronous buckets, RING_FREE when idle
    u32 ring_mask = 0;
    u32* d_aq = nullptr;    // ring counters
    HubRec* d_hubs = nullptr;  // hub records of the grid tier
    u32 hub_cap = 0;
    Ctl* d_ctl = nullptr;
    Ctl* h_ctl_init = nullptr;  // pinned: the control block every run starts from
    Ctl* h_ctl_out = nullptr;   // pinned: the control block every run ends with
    std::vector<void*> allocs;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int captured_mode = MODE_DELTA;
    u32 captured_delta = 0;
    u32 epoch_hint = 1;

    template <class T>
    pfg_status dalloc(T** p, u64 count) {
        void* q = nullptr;
        const u64 b = std::max<u64>(1, count) * sizeof(T);
        cudaError_t e = cudaMalloc(&q, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(PFG_ERR_OUT_OF_MEMORY, "cudaMalloc of %.1f MB failed: %s", b / 1048576.0,
                             cudaGetErrorString(e));
        }
        allocs.push_back(q);
        bytes += b;
        *p = (T*)q;
        return PFG_OK;
    }
};

static void drop_graph(pfg_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

extern "C" void pfg_batch_destroy(pfg_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (void* p : b->allocs) cudaFree(p);
    if (b->h_ctl_init) cudaFreeHost(b->h_ctl_init);
    if (b->h_ctl_out) cudaFreeHost(b->h_ctl_out);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    cudaGetLastError();
    delete b;
}

#define B_CUDA(call)                                                                           \
    do {                                                                                       \
        cudaError_t e__ = (call);                                                              \
        if (e__ != cudaSuccess) {                                                              \
            cudaGetLastError();                                                                \
            return set_error(e__ == cudaErrorMemoryAllocation ? PFG_ERR_OUT_OF_MEMORY : PFG_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e__));                 \
        }                                                                                      \
    } while (0)

static pfg_status batch_create(pfg_batch* b, uint32_t num_graphs, const uint32_t* const* rows,
                               const uint32_t* const* cols, const uint32_t* const* ws,
                               const uint32_t* ns, const uint32_t* ms) {
    // Validate every graph and lay out their padded rows back to back.
    std::vector<std::vector<u32>> prows(num_graphs);
    u64 pad_total = 0, rows_total = 0, m_total = 0, n_total = 0;
    double w_sum = 0.0;
    for (u32 g = 0; g < num_graphs; ++g) {
        u32 mw = 0;
        pfg_status st = validate_csr(rows[g], cols[g], ws[g], ns[g], ms[g], &mw);
        if (st != PFG_OK) return st;
        b->maxw = std::max(b->maxw, mw);
        for (u32 u = 0; u < ns[g]; ++u) {
            const u32 deg = rows[g][u + 1] - rows[g][u];
            b->max_deg = std::max(b->max_deg, deg);
            b->hub_rows += deg > 256u ? 1u : 0u;
        }
    }
    // no row with more than 4 arcs in any graph: every row gets exactly 4 slots
    // (row u of a graph starts at its first row + 4u; the kernel loads no prow)
    const bool uniform_rows = b->max_deg <= ROW_ALIGN;
    b->row_stride = uniform_rows ? ROW_ALIGN : 0u;
    for (u32 g = 0; g < num_graphs; ++g) {
        for (u32 k = 0; k < ms[g]; ++k) w_sum += ws[g][k];
        m_total += ms[g];
        n_total += ns[g];
        std::vector<u32>& pr = prows[g];
        pr.resize((size_t)ns[g] + 1);
        for (u32 u = 0; u < ns[g]; ++u) {
            pr[u] = (u32)pad_total;
            const u32 deg = rows[g][u + 1] - rows[g][u];
            pad_total += uniform_rows ? ROW_ALIGN : (u64)((deg + ROW_ALIGN - 1) / ROW_ALIGN) * ROW_ALIGN;
        }
        pr[ns[g]] = (u32)pad_total;
        if (pad_total >= 0xFFFFFFF0ull) return set_error(PFG_ERR_INVALID_GRAPH, "padded arcs of the batch exceed 2^32");
        b->g_n.push_back(ns[g]);
        b->g_m.push_back(ms[g]);
        b->g_rowbase.push_back((u32)rows_total);
        rows_total += (u64)ns[g] + 1;
    }
    b->avg_w = m_total ? w_sum / (double)m_total : 0.0;
    b->avg_deg = n_total ? (double)m_total / (double)n_total : 0.0;

    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || b->device < 0 || b->device >= count) {
        cudaGetLastError();
        return set_error(PFG_ERR_NO_DEVICE, "CUDA device %d not available", b->device);
    }
    B_CUDA(cudaSetDevice(b->device));
    B_CUDA(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device));
    const u64 S = b->max_states;
    const u64 need = pad_total * 8 + rows_total * 4 + S * 8 + 8 * S * 4 + 3ull * b->max_inst * 4;
    size_t free_b = 0, total_b = 0;
    B_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (need > free_b)
        return set_error(PFG_ERR_OUT_OF_MEMORY, "Not enough GPU memory: need %.1f MB, free %.1f MB",
                         need / 1048576.0, free_b / 1048576.0);
    B_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    B_CUDA(cudaEventCreate(&b->ev0));
    B_CUDA(cudaEventCreate(&b->ev1));

    auto t0 = std::chrono::steady_clock::now();
    pfg_status st = b->dalloc(&b->d_adj, pad_total);
    if (st == PFG_OK) st = b->dalloc(&b->d_prow, rows_total);
    if (st != PFG_OK) return st;
    // Every copy is ordered on the batch's stream, before the kernel that reads
    // it: the stream does not synchronise with the legacy default stream, and a
    // pageable cudaMemcpy may return before its DMA has landed.
    for (u32 g = 0; g < num_graphs; ++g) {
        const u32 n = ns[g], m = ms[g];
        u32 *d_row = nullptr, *d_col = nullptr, *d_w = nullptr;
        B_CUDA(cudaMemcpyAsync(b->d_prow + b->g_rowbase[g], prows[g].data(), ((size_t)n + 1) * 4,
                               cudaMemcpyHostToDevice, b->stream));
        B_CUDA(cudaMalloc((void**)&d_row, ((size_t)n + 1) * 4));
        cudaError_t e = cudaMalloc((void**)&d_col, std::max<size_t>(1, (size_t)m) * 4);
        if (e == cudaSuccess) e = cudaMalloc((void**)&d_w, std::max<size_t>(1, (size_t)m) * 4);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_row, rows[g], ((size_t)n + 1) * 4, cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess && m) e = cudaMemcpyAsync(d_col, cols[g], (size_t)m * 4, cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess && m) e = cudaMemcpyAsync(d_w, ws[g], (size_t)m * 4, cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = launch_build_adj(d_row, d_col, d_w, b->d_prow + b->g_rowbase[g], n, b->d_adj, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        cudaFree(d_row);
        if (d_col) cudaFree(d_col);
        if (d_w) cudaFree(d_w);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(PFG_ERR_CUDA, "batch upload of graph %u failed: %s", g, cudaGetErrorString(e));
        }
    }
    b->upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    st = b->dalloc(&b->d_state, S);
    for (int i = 0; i < 5 && st == PFG_OK; ++i) st = b->dalloc(&b->d_q[i], S);
    for (int i = 0; i < 3 && st == PFG_OK; ++i) st = b->dalloc(&b->d_stamp[i], S);
    if (st == PFG_OK) st = b->dalloc(&b->d_inst_off, (u64)b->max_inst + 1);
    if (st == PFG_OK) st = b->dalloc(&b->d_inst_rowbase, b->max_inst);
    if (st == PFG_OK) st = b->dalloc(&b->d_srcs, b->max_inst);
    if (st == PFG_OK) st = b->dalloc(&b->d_ctl, 1);
    u64 ring = 1024;  // room for two entries per state (one per strict improvement in flight)
    while (ring < 2 * (u64)S && ring < (1ull << 32)) ring <<= 1;
    if (st == PFG_OK) st = b->dalloc(&b->d_ring, ring);
    if (st == PFG_OK) st = b->dalloc(&b->d_aq, (u64)AQ_WORDS);
    if (st != PFG_OK) return st;
    b->ring_mask = (u32)(ring - 1);
    if (b->hub_rows) {
        // instances may repeat a graph: bound by the states, a hub row has > 256 arcs
        b->hub_cap = (u32)std::min<u64>(std::max<u64>(1024, 2 * b->hub_rows * std::max<u64>(1, b->max_inst)), 1u << 24);
        st = b->dalloc(&b->d_hubs, (u64)b->hub_cap);
        if (st != PFG_OK) return st;
        B_CUDA(cudaMemsetAsync(b->d_hubs, 0, (size_t)b->hub_cap * sizeof(HubRec), b->stream));
    }
    B_CUDA(cudaMemsetAsync(b->d_ring, 0xFF, ring * 8, b->stream));
    B_CUDA(cudaMemsetAsync(b->d_aq, 0, AQ_WORDS * 4, b->stream));
    for (int i = 0; i < 3; ++i) B_CUDA(cudaMemsetAsync(b->d_stamp[i], 0, S * 4, b->stream));
    B_CUDA(cudaMallocHost((void**)&b->h_ctl_init, sizeof(Ctl)));
    B_CUDA(cudaMallocHost((void**)&b->h_ctl_out, sizeof(Ctl)));
    memset(b->h_ctl_init, 0, sizeof(Ctl));
    memset(b->h_ctl_out, 0, sizeof(Ctl));
    Ctl c0;
    memset(&c0, 0, sizeof(c0));
    c0.near_epoch = c0.far_epoch = c0.r_epoch = 1;
    B_CUDA(cudaMemcpyAsync(b->d_ctl, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, b->stream));
    B_CUDA(cudaStreamSynchronize(b->stream));
    return PFG_OK;
}

extern "C" pfg_status pfg_batch_create(uint32_t num_graphs, const uint32_t* const* row_offsets,
                                       const uint32_t* const* col_indices,
                                       const uint32_t* const* weights, const uint32_t* n,
                                       const uint32_t* m, uint64_t max_states,
                                       uint32_t max_instances, int32_t device, pfg_batch** out) {
    if (!out || !row_offsets || !col_indices || !weights || !n || !m || num_graphs == 0)
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_batch_create: NULL argument or no graphs");
    *out = nullptr;
    if (max_instances == 0 || max_states == 0 || max_states >= 0xFFFFFFFFull)
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_batch_create: need 0 < max_states < 2^32 and max_instances > 0");
    pfg_batch* b = new pfg_batch();
    b->device = device;
    b->num_graphs = num_graphs;
    b->max_states = max_states;
    b->max_inst = max_instances;
    pfg_status st = batch_create(b, num_graphs, row_offsets, col_indices, weights, n, m);
    if (st != PFG_OK) {
        pfg_batch_destroy(b);
        return st;
    }
    *out = b;
    return PFG_OK;
}

extern "C" pfg_status pfg_batch_set_instances(pfg_batch* b, const uint32_t* inst_graph,
                                              const uint32_t* inst_src, uint32_t count) {
    if (!b || !inst_graph || !inst_src) return set_error(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (count == 0 || count > b->max_inst) return set_error(PFG_ERR_INVALID_ARGUMENT, "invalid batch size");
    std::vector<u32> off(count + 1), rb(count);
    u64 acc = 0;
    for (u32 i = 0; i < count; ++i) {
        const u32 g = inst_graph[i];
        if (g >= b->num_graphs) return set_error(PFG_ERR_INVALID_ARGUMENT, "instance %u: graph %u out of range", i, g);
        if (inst_src[i] >= b->g_n[g]) return set_error(PFG_ERR_INVALID_ARGUMENT, "source out of range");
        off[i] = (u32)acc;
        rb[i] = b->g_rowbase[g];
        acc += b->g_n[g];
        if (acc > b->max_states)
            return set_error(PFG_ERR_CAPACITY, "instances need %llu state words, the batch holds %llu",
                             (unsigned long long)acc, (unsigned long long)b->max_states);
    }
    off[count] = (u32)acc;
    B_CUDA(cudaSetDevice(b->device));
    B_CUDA(cudaStreamSynchronize(b->stream));
    // ordered on the batch's stream, which does not wait for the legacy stream
    B_CUDA(cudaMemcpyAsync(b->d_inst_off, off.data(), ((size_t)count + 1) * 4, cudaMemcpyHostToDevice, b->stream));
    B_CUDA(cudaMemcpyAsync(b->d_inst_rowbase, rb.data(), (size_t)count * 4, cudaMemcpyHostToDevice, b->stream));
    B_CUDA(cudaMemcpyAsync(b->d_srcs, inst_src, (size_t)count * 4, cudaMemcpyHostToDevice, b->stream));
    B_CUDA(cudaStreamSynchronize(b->stream));
    b->inst_off = off;
    b->num_inst = count;
    b->total_states = acc;
    drop_graph(b);  // a recorded run refers to the old table size
    return PFG_OK;
}

// Fills the initial control block and the kernel parameters of one run.
static pfg_status batch_prepare(pfg_batch* b, const pfg_options* opt_in, RunParams& p, int& grid,
                                int& block, pfg_options& o, int& mode, u32& delta) {
    if (b->num_inst == 0) return set_error(PFG_ERR_INVALID_ARGUMENT, "no instances set");
    o = opt_in ? *opt_in : default_options();
    sanitize_options(o);
    if (o.algo == PFG_ALGO_NAIVE) o.algo = PFG_ALGO_DELTA;  // as the reference does for batches
    if (o.policy == PFG_POLICY_LEARNED)
        return set_error(PFG_ERR_INVALID_ARGUMENT, "the learned policy runs on single-graph solvers");
    mode = o.algo == PFG_ALGO_FRONTIER ? MODE_FRONTIER : MODE_DELTA;
    delta = mode == MODE_DELTA ? (o.delta ? o.delta : auto_delta_of(b->avg_w, b->avg_deg)) : 0u;
    if (b->epoch_hint >= 0xF0000000u) {
        for (int i = 0; i < 3; ++i) B_CUDA(cudaMemsetAsync(b->d_stamp[i], 0, b->max_states * 4, b->stream));
        Ctl c0;
        memset(&c0, 0, sizeof(c0));
        c0.near_epoch = c0.far_epoch = c0.r_epoch = 1;
        B_CUDA(cudaMemcpyAsync(b->d_ctl, &c0, sizeof(Ctl), cudaMemcpyHostToDevice, b->stream));
        B_CUDA(cudaStreamSynchronize(b->stream));
        b->epoch_hint = 1;
    }
    Ctl* c = b->h_ctl_init;
    memset(c, 0, offsetof(Ctl, persist));
    c->rd.phase = PH_INIT;
    c->rd.map_mode = 1u;
    c->far_min[0] = c->far_min[1] = ~0ull;
    u32 max_n = 0;
    for (u32 x : b->g_n) max_n = std::max(max_n, x);
    c->round_cap = (u32)std::min<u64>(4ull * max_n + 1000ull, 0x7FFFFFFFull);
    c->rd.delta = delta ? delta : 1u;
    c->delta0 = delta;
    c->rd.heavy = (mode == MODE_DELTA && delta < b->maxw) ? 1u : 0u;

    memset(&p, 0, sizeof(p));
    p.adj = b->d_adj;
    p.prow = b->d_prow;
    p.row_stride = b->row_stride;
    p.short_rows = b->max_deg <= 32u ? 1u : 0u;
    p.n = (u32)std::min<u64>(b->total_states, 0xFFFFFFFFull);
    p.maxw = b->maxw;
    p.avg_w = b->avg_w;
    p.avg_deg = b->avg_deg;
    p.k = b->num_inst;
    p.total = (u32)b->total_states;
    p.srcs = b->d_srcs;
    p.inst_off = b->d_inst_off;
    p.inst_rowbase = b->d_inst_rowbase;
    p.state = b->d_state;
    p.nearq[0] = b->d_q[0];
    p.nearq[1] = b->d_q[1];
    p.farq[0] = b->d_q[2];
    p.farq[1] = b->d_q[3];
    p.rq = b->d_q[4];
    p.near_stamp = b->d_stamp[0];
    p.far_stamp = b->d_stamp[1];
    p.r_stamp = b->d_stamp[2];
    p.ctl = b->d_ctl;
    p.delta = delta ? delta : 1u;
    p.mode = mode;
    p.prefix_scan = (mode == MODE_FRONTIER && o.compaction == PFG_COMPACT_PREFIX_SCAN) ? 1 : 0;
    p.eager = eager_rounds_for(o);
    if (o.eager < 0 && b->avg_deg > 6.0) p.eager = 0;  // as the single-graph solver: road-like graphs only
    p.timeout_ns = device_timeout_ns();
    if (async_buckets_for(o, mode)) {
        p.ring = b->d_ring;
        p.ring_mask = b->ring_mask;
        p.aq = b->d_aq;
    }
    block = o.block_size;
    if (b->d_hubs && o.mapping == PFG_MAP_HYBRID && b->max_deg > 8u * (u32)block) {
        p.hubs = b->d_hubs;
        p.hub_cap = b->hub_cap;
        p.hub_min = 8u * (u32)block;
        p.hub_chunk = 4u * (u32)block;
        p.aq = b->d_aq;
    }
    configure_drain(p, o.schedule, b->d_hubs, b->hub_cap, b->max_deg, b->d_aq, o.mapping, block);
    const int bps = blocks_per_sm_for(o, false, o.mapping);
    if (bps <= 0) return set_error(PFG_ERR_CUDA, "occupancy query failed for block size %d", block);
    grid = b->sm_count * bps;
    p.eager_max_items = (u32)std::max<long long>(1, (long long)grid * block / 4);
    return PFG_OK;
}

static pfg_status batch_enqueue(pfg_batch* b, const RunParams& p, const pfg_options& o, int grid, int block) {
    B_CUDA(cudaMemcpyAsync(b->d_ctl, b->h_ctl_init, offsetof(Ctl, persist), cudaMemcpyHostToDevice, b->stream));
    cudaError_t e = launch_persistent(p, false, o.atomic, o.mapping, block, grid, b->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(PFG_ERR_CUDA, "persistent launch failed (grid %d x %d): %s", grid, block,
                         cudaGetErrorString(e));
    }
    B_CUDA(cudaMemcpyAsync(b->h_ctl_out, b->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, b->stream));
    return PFG_OK;
}

static pfg_status batch_complete(pfg_batch* b, int mode, u32 delta, pfg_stats* stats, float* ms) {
    B_CUDA(cudaStreamSynchronize(b->stream));
    const Ctl* c = b->h_ctl_out;
    b->epoch_hint = std::max({c->near_epoch, c->far_epoch, c->r_epoch});
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->edges_scanned = c->stats[0];
        stats->atomics_issued = c->stats[1];
        stats->updates = c->stats[2];
        stats->pushes = c->stats[3];
        stats->iterations = c->iterations;
        stats->host_syncs = 1;
        stats->launches = 1;
        stats->buckets = mode == MODE_DELTA ? c->buckets : 0u;
        stats->delta = delta;
        stats->rounds = c->rounds;
    }
    if (ms) {
        float t = 0.f;
        B_CUDA(cudaEventElapsedTime(&t, b->ev0, b->ev1));
        *ms = t;
    }
    switch (c->rd.status) {
        case DS_OK: return PFG_OK;
        case DS_BAD_SOURCE: return set_error(PFG_ERR_INVALID_ARGUMENT, "source out of range");
        case DS_NOT_CONVERGED: return set_error(PFG_ERR_NOT_CONVERGED, "batch did not converge");
        case DS_TIMEOUT:
            // the next run must find the ring empty
            cudaMemsetAsync(b->d_ring, 0xFF, ((u64)b->ring_mask + 1) * 8, b->stream);
            cudaMemsetAsync(b->d_aq, 0, AQ_WORDS * 4, b->stream);
            cudaStreamSynchronize(b->stream);
            return set_error(PFG_ERR_DEVICE_TIMEOUT, "device-side wait timed out: %s made no progress for %llu ms",
                             wait_site_name(c->wait_site), (unsigned long long)(device_timeout_ns() / 1000000ull));
        default: return set_error(PFG_ERR_CUDA, "device status %u", c->rd.status);
    }
}

extern "C" pfg_status pfg_batch_run(pfg_batch* b, const pfg_options* opt, pfg_stats* stats, float* ms) {
    if (!b) return set_error(PFG_ERR_INVALID_ARGUMENT, "batch is NULL");
    B_CUDA(cudaSetDevice(b->device));
    RunParams p;
    pfg_options o;
    int grid = 0, block = 0, mode = 0;
    u32 delta = 0;
    pfg_status st = batch_prepare(b, opt, p, grid, block, o, mode, delta);
    if (st != PFG_OK) return st;
    B_CUDA(cudaEventRecord(b->ev0, b->stream));
    st = batch_enqueue(b, p, o, grid, block);
    if (st != PFG_OK) return st;
    B_CUDA(cudaEventRecord(b->ev1, b->stream));
    return batch_complete(b, mode, delta, stats, ms);
}

extern "C" pfg_status pfg_batch_capture(pfg_batch* b, const pfg_options* opt) {
    if (!b) return set_error(PFG_ERR_INVALID_ARGUMENT, "batch is NULL");
    B_CUDA(cudaSetDevice(b->device));
    B_CUDA(cudaStreamSynchronize(b->stream));
    drop_graph(b);
    RunParams p;
    pfg_options o;
    int grid = 0, block = 0, mode = 0;
    u32 delta = 0;
    pfg_status st = batch_prepare(b, opt, p, grid, block, o, mode, delta);
    if (st != PFG_OK) return st;
    B_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    st = batch_enqueue(b, p, o, grid, block);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st != PFG_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(PFG_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    }
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        cudaGetLastError();
        return set_error(PFG_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    }
    b->graph = g;
    b->captured_mode = mode;
    b->captured_delta = delta;
    return PFG_OK;
}

extern "C" pfg_status pfg_batch_replay(pfg_batch* b, pfg_stats* stats, float* ms) {
    if (!b || !b->exec) return set_error(PFG_ERR_INVALID_ARGUMENT, "no captured run");
    B_CUDA(cudaSetDevice(b->device));
    B_CUDA(cudaEventRecord(b->ev0, b->stream));
    B_CUDA(cudaGraphLaunch(b->exec, b->stream));
    B_CUDA(cudaEventRecord(b->ev1, b->stream));
    return batch_complete(b, b->captured_mode, b->captured_delta, stats, ms);
}

extern "C" uint64_t pfg_batch_instance_offset(const pfg_batch* b, uint32_t inst) {
    if (!b || inst > b->num_inst) return 0;
    return b->inst_off[inst];
}
extern "C" uint64_t pfg_batch_num_states(const pfg_batch* b) { return b ? b->total_states : 0; }
extern "C" void* pfg_batch_stream(const pfg_batch* b) { return b ? (void*)b->stream : nullptr; }
extern "C" double pfg_batch_upload_ms(const pfg_batch* b) { return b ? b->upload_ms : 0.0; }
extern "C" uint64_t pfg_batch_device_bytes(const pfg_batch* b) { return b ? b->bytes : 0; }

extern "C" pfg_status pfg_batch_copy_state(pfg_batch* b, uint64_t first, uint64_t count, uint64_t* h_out) {
    if (!b || !h_out) return set_error(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (first > b->total_states || count > b->total_states - first)  // (no sum that can wrap)
        return set_error(PFG_ERR_INVALID_ARGUMENT, "range outside the state");
    B_CUDA(cudaSetDevice(b->device));
    B_CUDA(cudaMemcpyAsync(h_out, b->d_state + first, count * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CUDA(cudaStreamSynchronize(b->stream));
    return PFG_OK;
}
