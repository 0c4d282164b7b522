// pfg_internal.h - host helpers shared by the solver, batch and serving entry
// points of libpfg_b200.so (not part of the C ABI).
#pragma once
#include "../../include/pfg.h"
#include "pfg_common.cuh"

#include <cuda_runtime.h>

#include <algorithm>

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
int blocks_per_sm_for(const pfg_options& o, bool astar, int map, bool iw = false, u32 k = 0);

// Eager sub-rounds per grid round of the hybrid mapping when the caller leaves
// the choice to the engine (pfg_options::eager < 0), and the average degree
// above which the engine turns them off (hubs make in-round propagation redundant).
constexpr int kDefaultEager = 4;
constexpr double kEagerMaxAvgDegree = 6.0;

// Eager sub-rounds when the caller leaves the choice to the engine.
u32 eager_rounds_for(const pfg_options& o);

// Milliseconds from the PFG_TIMEOUT_MS environment variable (default 2000)
// as the bound of every device-side wait, in nanoseconds.
u64 device_timeout_ns();

// Whether a run drains its buckets asynchronously (ring queue + claimed lists).
bool async_buckets_for(const pfg_options& o, int mode);

// Asynchronous drains: warp workers for PFG_SCHEDULE_WARP with the Hybrid
// mapping, else block-synchronous passes over each CTA's claimed list. Sets
// RunParams::warp_drain and the warp tier of long rows, and enables the hub
// records (hubs, hub_cap) for the rows beyond the CTA tier.
void configure_drain(RunParams& p, int schedule, HubRec* hubs, u32 hub_cap, u32 max_deg, u32* aq, int mapping,
                     int block);

}  // namespace pfg

#include <string>
#include <vector>

// One solver: the graph and the working set of max_batch instances on one device.
struct pfg_solver {
    typedef pfg::u32 u32;
    typedef pfg::u64 u64;
    typedef pfg::Ctl Ctl;
    typedef pfg::PolicyNet PolicyNet;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    u32 n = 0, m = 0, K = 1, maxw = 0;
    u32 max_deg = 0;            // largest out-degree
    u32 row_stride = 0;         // ROW_ALIGN when every row has exactly ROW_ALIGN slots, else 0
    u64 hub_rows = 0;           // vertices with more than 256 arcs
    u64 m_pad = 0;
    double hscale = 0.0, avg_w = 0.0, avg_deg = 0.0;
    bool has_xy = false;
    std::vector<double> hx, hy;  // host copies of the coordinates (A* target lookup)
    int sm_count = 1;
    double upload_ms = 0.0;
    u64 bytes = 0;

    uint2* d_adj = nullptr;
    u32* d_prow = nullptr;
    double* d_x = nullptr;
    double* d_y = nullptr;
    u64* d_state = nullptr;
    u32* d_q[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // near0, near1, far0, far1, R
    u32* d_stamp[3] = {nullptr, nullptr, nullptr};                // near, far, R
    u32* d_naive[2] = {nullptr, nullptr};
    unsigned long long* d_ring = nullptr;  // ring queue of asynchronous buckets [ring_mask + 1], RING_FREE when idle
    u32 ring_mask = 0;
    u32* d_aq = nullptr;        // ring counters [AQ_WORDS]
    u32* d_iw = nullptr;        // independent-window block [iw_words(min(K, IW_MAX_INST))]
    pfg::HubRec* d_hubs = nullptr;  // hub records of the grid tier [hub_cap]
    u32 hub_cap = 0;
    u32* d_srcs = nullptr;
    u32* d_path = nullptr;      // path extraction scratch [n + 1]
    u32* d_path_len = nullptr;
    Ctl* d_ctl = nullptr;
    PolicyNet* d_net = nullptr;
    bool has_net = false;
    float* d_trace = nullptr;   // per-bucket policy features of traced runs
    u32 trace_cap = 0;

    Ctl* h_ctl = nullptr;       // pinned mirror of the control block
    u32* h_srcs = nullptr;      // pinned staging of the sources [K]

    // streamed multi-source runs (pfg_run_dist_async): the distances of one run
    // are split into d_dist and copied on copy_stream while the next run computes
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_split = nullptr, ev_copied = nullptr;
    u32* d_dist = nullptr;        // [K n], allocated on first use
    uint32_t* pipe_out = nullptr; // host buffer of the streamed run in flight (its copy not started)
    u32 pipe_k = 0;
    bool pipe_copying = false;    // a copy may be in flight on copy_stream

    // last asynchronous run
    bool pending = false;
    pfg_status pending_status = PFG_OK;
    int last_mode = pfg::MODE_DELTA;
    u32 last_delta = 0;
    u32 last_k = 0;
    bool last_iw = false; // the run in flight uses independent bucket windows
    u32 epoch_hint = 1;   // largest epoch known to the host (stamps reset near 2^32)
    std::vector<void*> allocs;

    template <class T>
    pfg_status dalloc(T** p, u64 count) {
        void* q = nullptr;
        const u64 b = std::max<u64>(1, count) * sizeof(T);
        cudaError_t e = cudaMalloc(&q, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return pfg::set_error(PFG_ERR_OUT_OF_MEMORY, "cudaMalloc of %.1f MB failed: %s", b / 1048576.0,
                        cudaGetErrorString(e));
        }
        allocs.push_back(q);
        bytes += b;
        *p = (T*)q;
        return PFG_OK;
    }
};
