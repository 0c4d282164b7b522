// pfg_serve.cu - continuous batching of point-to-point A* queries.
//
// The graph and the working set stay resident. A query occupies one of S
// slots (slot i owns state words [i*n, (i+1)*n)). All slots share one
// Delta-stepping machine in one persistent kernel: slot i's keys are
// dist + h_i(v) + phi_i with phi_i chosen at admission so that the query
// enters at the start of the next bucket, which lets queries that arrive at
// different times share one monotone bucket sequence without holding up the
// ones in flight. The host drives bounded steps: admit waiting queries into
// free slots, run at most R rounds, collect the slots whose far pile went
// empty at a bucket advance (their target distance is final), repeat. With
// asynchronous buckets (the default schedule) a step's budget counts bucket
// drains: one barrier epoch per bucket.
// The reference answers one query per GpuSolver::astar call
// (src/gpu_sssp.cu:549-551); results here are the same distances.
#include "../../include/pfg.h"
#include "pfg_common.cuh"
#include "pfg_internal.h"
#include "pfg_kernels.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <vector>

using namespace pfg;

namespace {

// Most slots an automatically sized server takes (slots = 0 at creation).
constexpr u64 kMaxAutoSlots = 2048;

struct Request {
    uint64_t id;
    uint32_t src, dst;
    double submit_us;
};

struct SlotInfo {
    bool used = false;
    Request req{};
    double admit_us = 0.0;
    uint32_t admit_round = 0;
};

// State words of the admitted slots back to (INF, NO_PARENT): blockIdx.y is the
// admitted slot, the x blocks stream its n words with 16-byte stores (a slot's
// range starts at a multiple of n words, so its first word may sit mid-pair).
__global__ void k_serve_clear(u64* state, const u32* slots, u32 n) {
    u64* base = state + (u64)slots[blockIdx.y] * n;
    const u32 head = (u32)(((uintptr_t)base >> 3) & 1u);  // one word up to a 16-byte boundary
    const u32 stride = gridDim.x * blockDim.x;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (head && t == 0 && n > 0) base[0] = STATE_INIT;
    const u32 body = n > head ? (n - head) / 2u : 0u;
    ulonglong2* v = reinterpret_cast<ulonglong2*>(base + head);
    for (u32 i = t; i < body; i += stride) v[i] = make_ulonglong2(STATE_INIT, STATE_INIT);
    const u32 tail = head + 2u * body;
    if (t == 0 && tail < n) base[tail] = STATE_INIT;
}

struct AdmitParams {
    Ctl* ctl;
    u64* state;
    u32* nearq0;
    u32* farq[2];
    u32* far_stamp;
    const double* x;
    const double* y;
    double hscale;
    int use_h;
    u32 n;
    u32 delta;
    u32 maxw;
    u32 step_rounds;
    const u32* adm_slot;
    const u32* adm_src;
    const u32* adm_dst;
    u32 m;
    u32* target;
    double* tx;
    double* ty;
    long long* phi;
    u32* far_cnt;
    u32* active;
    u32* done;
    u32* aq;     // ring counters (asynchronous buckets), else nullptr
    u32 grid;    // CTAs of the persistent launch
};

// Admission and step preparation, one thread: seeds the admitted slots and
// sets the machine up to run (restarts an idle machine, or resumes a paused one).
__global__ void k_serve_begin_step(AdmitParams a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Ctl* c = a.ctl;
    Rd& r = c->rd;
    const bool idle = r.phase == PH_DONE;
    if (a.m > 0 && idle) {
        // Fresh bucket sequence starting at key 0; new stamp epochs make every
        // old stamp word stale.
        r.phase = PH_LIGHT;
        r.status = DS_OK;
        r.in_buf = 0u;
        r.in_count = a.m;
        r.far_in = 0u;
        r.far_out = 0u;
        r.delta = a.delta;
        r.heavy = a.delta < a.maxw ? 1u : 0u;
        r.lo = 0ull;
        r.hi = a.delta;
        r.near_epoch += 1u;
        r.far_epoch += 1u;
        r.r_epoch += 1u;
        c->near_epoch = r.near_epoch;
        c->far_epoch = r.far_epoch;
        c->r_epoch = r.r_epoch;
        c->cnt[C_NEAR0] = a.m;
        c->cnt[C_NEAR1] = 0u;
        c->cnt[C_FAR0] = c->cnt[C_FAR1] = 0u;
        c->cnt[C_R] = 0u;
        c->far_min[0] = c->far_min[1] = ~0ull;
        r.async_bkt = 0u;
        if (a.aq) {
            // asynchronous first bucket: every CTA scans its slice of the seeds
            // in near queue 0, then drains the ring and its claimed list
            c->cnt[C_NEAR0] = 0u;
            r.in_kind = 1u;
            r.async_bkt = 1u;
            r.phase = PH_ASYNC;
            a.aq[AQ_HEAD] = 0u;
            a.aq[AQ_TAIL] = 0u;
            a.aq[AQ_DONE] = 0u;
            a.aq[AQ_BUSY] = a.grid;
            a.aq[AQ_IDLE] = 0u;
        }
    }
    for (u32 j = 0; j < a.m; ++j) {
        const u32 s = a.adm_slot[j], src = a.adm_src[j], dst = a.adm_dst[j];
        const u32 gi = s * a.n + src;
        a.state[gi] = pack_state(0u, NO_PARENT);
        double xt = 0.0, yt = 0.0;
        u32 h = 0;
        if (a.use_h) {
            xt = a.x[dst];
            yt = a.y[dst];
            h = heuristic_value(a.x[src], a.y[src], xt, yt, a.hscale);
        }
        a.target[s] = dst;
        a.tx[s] = xt;
        a.ty[s] = yt;
        a.active[s] = 1u;
        a.done[s] = 0u;
        if (idle) {
            // key of the seed = start of the fresh window
            a.phi[s] = (long long)r.lo - (long long)h;
            a.nearq0[j] = gi;
            a.far_cnt[s] = 0u;
        } else {
            // key of the seed = start of the next bucket: wait in the far pile
            a.phi[s] = (long long)r.hi - (long long)h;
            const u32 fo = r.far_out;
            if (atomicExch(a.far_stamp + gi, r.far_epoch) != r.far_epoch) {
                a.farq[fo][c->cnt[C_FAR0 + fo]] = gi;
                c->cnt[C_FAR0 + fo] += 1u;
            }
            if (r.hi < c->far_min[fo]) c->far_min[fo] = r.hi;
            a.far_cnt[s] = 1u;
        }
    }
    if (r.phase == PH_PAUSE) r.phase = c->resume_phase;
    c->bar_count = 0u;
    c->bar_gen = 0u;
    c->step_left = a.step_rounds;
    // A server runs for ever; each step is bounded by step_rounds instead, so the
    // run-level round cap only has to outlast the counter.
    c->round_cap = 0x7FFFFFFFu;
    if (c->rounds > 0x3FFFFFFFu) c->rounds = 0u;
    __threadfence();
}

// Target state word of every finished slot (others: ~0).
__global__ void k_serve_collect(const u64* state, u32 n, const u32* target, const u32* done, u32 S, u64* out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S) out[i] = done[i] ? state[(u64)i * n + target[i]] : ~0ull;
}

__global__ void k_serve_init(Ctl* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) c->rd.phase = PH_DONE;
}

}  // namespace

struct pfg_server {
    pfg_solver* s = nullptr;
    u32 S = 0;
    pfg_options opt{};
    u32 delta = 0;
    int grid = 0, block = 0;
    u32* d_target = nullptr;
    double* d_tx = nullptr;
    double* d_ty = nullptr;
    long long* d_phi = nullptr;
    u32* d_far_cnt = nullptr;
    u32* d_active = nullptr;
    u32* d_done = nullptr;
    u32* d_adm = nullptr;   // [3 * S]: slots, sources, targets
    u64* d_out = nullptr;
    u32* h_adm = nullptr;   // pinned [3 * S]
    u64* h_out = nullptr;   // pinned [S]
    u32* h_done = nullptr;  // pinned [S]
    Rd* h_rd = nullptr;     // pinned
    u32* h_rounds = nullptr;
    std::deque<Request> pending;
    std::vector<SlotInfo> slots;
    std::vector<pfg_query_result> results;
    uint64_t next_id = 1;
    std::chrono::steady_clock::time_point t0;
    u64 steps = 0;

    double now_us() const {
        return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    }
};

#define S_CUDA(call)                                                                            \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess) {                                                               \
            cudaGetLastError();                                                                 \
            return set_error(e__ == cudaErrorMemoryAllocation ? PFG_ERR_OUT_OF_MEMORY : PFG_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e__));                  \
        }                                                                                       \
    } while (0)

extern "C" void pfg_server_destroy(pfg_server* v) {
    if (!v) return;
    if (v->s) {
        cudaSetDevice(v->s->device);
        cudaStreamSynchronize(v->s->stream);
    }
    void* dev[] = {v->d_target, v->d_tx, v->d_ty, v->d_phi, v->d_far_cnt, v->d_active, v->d_done, v->d_adm, v->d_out};
    for (void* p : dev)
        if (p) cudaFree(p);
    void* host[] = {v->h_adm, v->h_out, v->h_done, v->h_rd, v->h_rounds};
    for (void* p : host)
        if (p) cudaFreeHost(p);
    if (v->s) pfg_destroy(v->s);
    cudaGetLastError();
    delete v;
}

static pfg_status server_setup(pfg_server* v) {
    const u32 S = v->S;
    S_CUDA(cudaSetDevice(v->s->device));
    S_CUDA(cudaMalloc((void**)&v->d_target, S * 4));
    S_CUDA(cudaMalloc((void**)&v->d_tx, S * 8));
    S_CUDA(cudaMalloc((void**)&v->d_ty, S * 8));
    S_CUDA(cudaMalloc((void**)&v->d_phi, S * 8));
    S_CUDA(cudaMalloc((void**)&v->d_far_cnt, S * 4));
    S_CUDA(cudaMalloc((void**)&v->d_active, S * 4));
    S_CUDA(cudaMalloc((void**)&v->d_done, S * 4));
    S_CUDA(cudaMalloc((void**)&v->d_adm, 3 * S * 4));
    S_CUDA(cudaMalloc((void**)&v->d_out, S * 8));
    // cleared on the solver's stream, which does not wait for the legacy stream
    cudaStream_t st0 = v->s->stream;
    S_CUDA(cudaMemsetAsync(v->d_target, 0, S * 4, st0));
    S_CUDA(cudaMemsetAsync(v->d_far_cnt, 0, S * 4, st0));
    S_CUDA(cudaMemsetAsync(v->d_active, 0, S * 4, st0));
    S_CUDA(cudaMemsetAsync(v->d_done, 0, S * 4, st0));
    S_CUDA(cudaMemsetAsync(v->d_phi, 0, S * 8, st0));
    S_CUDA(cudaMemsetAsync(v->d_tx, 0, S * 8, st0));
    S_CUDA(cudaMemsetAsync(v->d_ty, 0, S * 8, st0));
    S_CUDA(cudaMallocHost((void**)&v->h_adm, 3 * S * 4));
    S_CUDA(cudaMallocHost((void**)&v->h_out, S * 8));
    S_CUDA(cudaMallocHost((void**)&v->h_done, S * 4));
    S_CUDA(cudaMallocHost((void**)&v->h_rd, sizeof(Rd)));
    S_CUDA(cudaMallocHost((void**)&v->h_rounds, 16));
    k_serve_init<<<1, 1, 0, v->s->stream>>>(v->s->d_ctl);
    S_CUDA(cudaGetLastError());
    S_CUDA(cudaStreamSynchronize(v->s->stream));
    v->slots.assign(S, SlotInfo());
    return PFG_OK;
}

extern "C" pfg_status pfg_server_create(const uint32_t* row, const uint32_t* col, const uint32_t* w,
                                        const double* x, const double* y, uint32_t n, uint32_t m,
                                        double h_scale, double avg_w, double avg_deg, uint32_t slots,
                                        const pfg_options* opt, int32_t device, pfg_server** out) {
    if (!out || n == 0) return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_server_create: bad argument");
    *out = nullptr;
    if (slots == 0) {
        // Admission by device memory: as many slots as fit in 60 % of the free
        // memory after the graph (per slot: the packed state, five queues, three
        // stamp words and its share of the power-of-two ring, of 2 entries per state).
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count || cudaSetDevice(device) != cudaSuccess) {
            cudaGetLastError();
            return set_error(PFG_ERR_NO_DEVICE, "CUDA device %d not available", device);
        }
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            return set_error(PFG_ERR_CUDA, "cudaMemGetInfo failed");
        }
        const u64 graph_b = 8ull * ((u64)m + 3ull * n) + 32ull * n;
        const double budget = 0.6 * (double)(free_b > graph_b ? free_b - graph_b : 0);
        auto bytes_for = [&](u64 S) {
            u64 ring = 1024;
            while (ring < 2 * S * n && ring < (1ull << 32)) ring <<= 1;
            return (double)S * n * 40.0 + (double)ring * 8.0;
        };
        const u64 cap = std::min<u64>(kMaxAutoSlots, (0xFFFFFFFEull / n));
        u64 S = 1;
        while (S < cap && bytes_for(S + 1) <= budget) ++S;
        slots = (u32)S;
    }
    pfg_server* v = new pfg_server();
    v->S = slots;
    v->t0 = std::chrono::steady_clock::now();
    pfg_status st = pfg_create_on_device(row, col, w, x, y, n, m, h_scale, avg_w, avg_deg, slots, device, &v->s);
    if (st != PFG_OK) {
        delete v;
        return st;
    }
    v->opt = opt ? *opt : default_options();
    sanitize_options(v->opt);
    v->opt.algo = PFG_ALGO_DELTA;
    v->delta = v->opt.delta ? v->opt.delta : auto_delta_of(avg_w, avg_deg);
    v->block = v->opt.block_size;
    const int bps = blocks_per_sm_for(v->opt, true, v->opt.mapping);
    if (bps <= 0) {
        pfg_server_destroy(v);
        return set_error(PFG_ERR_CUDA, "occupancy query failed");
    }
    v->grid = v->s->sm_count * bps;
    st = server_setup(v);
    if (st != PFG_OK) {
        pfg_server_destroy(v);
        return st;
    }
    *out = v;
    return PFG_OK;
}

extern "C" pfg_status pfg_server_submit(pfg_server* v, uint32_t src, uint32_t dst, uint64_t* id_out) {
    if (!v) return set_error(PFG_ERR_INVALID_ARGUMENT, "server is NULL");
    if (src >= v->s->n || dst >= v->s->n) return set_error(PFG_ERR_INVALID_ARGUMENT, "source or target out of range");
    Request r{v->next_id++, src, dst, v->now_us()};
    v->pending.push_back(r);
    if (id_out) *id_out = r.id;
    return PFG_OK;
}

extern "C" pfg_status pfg_server_step(pfg_server* v, uint32_t max_rounds, uint32_t* admitted_out,
                                      uint32_t* completed_out) {
    if (!v) return set_error(PFG_ERR_INVALID_ARGUMENT, "server is NULL");
    if (max_rounds == 0) return set_error(PFG_ERR_INVALID_ARGUMENT, "max_rounds must be > 0");
    pfg_solver* s = v->s;
    const u32 S = v->S, n = s->n;
    S_CUDA(cudaSetDevice(s->device));
    // ---- admission into free slots ----
    u32 m = 0;
    const double t_admit = v->now_us();
    for (u32 i = 0; i < S && !v->pending.empty(); ++i) {
        if (v->slots[i].used) continue;
        const Request r = v->pending.front();
        v->pending.pop_front();
        v->slots[i].used = true;
        v->slots[i].req = r;
        v->slots[i].admit_us = t_admit;
        v->h_adm[m] = i;
        v->h_adm[S + m] = r.src;
        v->h_adm[2 * S + m] = r.dst;
        ++m;
    }
    bool any_used = false;
    for (u32 i = 0; i < S; ++i) any_used = any_used || v->slots[i].used;
    if (!any_used) {
        if (admitted_out) *admitted_out = 0;
        if (completed_out) *completed_out = 0;
        return PFG_OK;
    }
    cudaStream_t st = s->stream;
    if (m > 0) {
        S_CUDA(cudaMemcpyAsync(v->d_adm, v->h_adm, 3 * S * 4, cudaMemcpyHostToDevice, st));
        const u32 bx = (u32)std::max<u64>(1, std::min<u64>(((u64)n / 2 + 255) / 256, (u64)s->sm_count * 2));
        k_serve_clear<<<dim3(bx, m), 256, 0, st>>>(s->d_state, v->d_adm, n);
        S_CUDA(cudaGetLastError());
    }
    AdmitParams a;
    memset(&a, 0, sizeof(a));
    a.ctl = s->d_ctl;
    a.state = s->d_state;
    a.nearq0 = s->d_q[0];
    a.farq[0] = s->d_q[2];
    a.farq[1] = s->d_q[3];
    a.far_stamp = s->d_stamp[1];
    a.x = s->d_x;
    a.y = s->d_y;
    a.hscale = s->hscale;
    a.use_h = (s->has_xy && s->hscale > 0.0) ? 1 : 0;
    a.n = n;
    a.delta = v->delta;
    a.maxw = s->maxw;
    a.step_rounds = max_rounds;
    a.adm_slot = v->d_adm;
    a.adm_src = v->d_adm + S;
    a.adm_dst = v->d_adm + 2 * S;
    a.m = m;
    a.target = v->d_target;
    a.tx = v->d_tx;
    a.ty = v->d_ty;
    a.phi = v->d_phi;
    a.far_cnt = v->d_far_cnt;
    a.active = v->d_active;
    a.done = v->d_done;
    const bool async = async_buckets_for(v->opt, MODE_DELTA);
    a.aq = async ? s->d_aq : nullptr;
    a.grid = (u32)v->grid;
    k_serve_begin_step<<<1, 32, 0, st>>>(a);
    S_CUDA(cudaGetLastError());

    // ---- one bounded step of the shared machine ----
    RunParams p;
    memset(&p, 0, sizeof(p));
    p.adj = s->d_adj;
    p.prow = s->d_prow;
    p.row_stride = s->row_stride;
    p.short_rows = s->max_deg <= 32u ? 1u : 0u;
    p.x = s->d_x;
    p.y = s->d_y;
    p.n = n;
    p.maxw = s->maxw;
    p.hscale = s->hscale;
    p.avg_w = s->avg_w;
    p.avg_deg = s->avg_deg;
    p.m = s->m;
    p.k = S;
    p.total = S * n;
    p.srcs = s->d_srcs;
    p.astar = 1;
    p.use_h = a.use_h;
    p.state = s->d_state;
    p.nearq[0] = s->d_q[0];
    p.nearq[1] = s->d_q[1];
    p.farq[0] = s->d_q[2];
    p.farq[1] = s->d_q[3];
    p.rq = s->d_q[4];
    p.near_stamp = s->d_stamp[0];
    p.far_stamp = s->d_stamp[1];
    p.r_stamp = s->d_stamp[2];
    p.ctl = s->d_ctl;
    p.delta = v->delta;
    p.mode = MODE_DELTA;
    // learned Delta when asked for and a network is loaded; the fixed automatic Delta otherwise
    p.policy = (v->opt.policy == PFG_POLICY_LEARNED && s->has_net) ? 1 : 0;
    p.net = s->d_net;
    p.inst_target = v->d_target;
    p.inst_tx = v->d_tx;
    p.inst_ty = v->d_ty;
    p.inst_phi = v->d_phi;
    p.inst_far_cnt = v->d_far_cnt;
    p.inst_active = v->d_active;
    p.inst_done = v->d_done;
    p.step_rounds = max_rounds;
    p.resume = 1;
    p.eager = eager_rounds_for(v->opt);
    if (v->opt.eager < 0 && s->avg_deg > 6.0) p.eager = 0;
    p.eager_max_items = (u32)std::max<long long>(1, (long long)v->grid * v->block / 4);
    p.timeout_ns = device_timeout_ns();
    if (async) {
        p.ring = s->d_ring;
        p.ring_mask = s->ring_mask;
        p.aq = s->d_aq;
    }
    configure_drain(p, v->opt.schedule, nullptr, 0u, s->max_deg, s->d_aq, v->opt.mapping, v->block);
    cudaError_t le = launch_persistent(p, true, v->opt.atomic, v->opt.mapping, v->block, v->grid, st);
    if (le != cudaSuccess) {
        cudaGetLastError();
        return set_error(PFG_ERR_CUDA, "serving step launch failed: %s", cudaGetErrorString(le));
    }
    k_serve_collect<<<(S + 127) / 128, 128, 0, st>>>(s->d_state, n, v->d_target, v->d_done, S, v->d_out);
    S_CUDA(cudaGetLastError());
    S_CUDA(cudaMemcpyAsync(v->h_out, v->d_out, S * 8, cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaMemcpyAsync(v->h_done, v->d_done, S * 4, cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaMemcpyAsync(v->h_rd, &s->d_ctl->rd, sizeof(Rd), cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaMemcpyAsync(v->h_rounds, &s->d_ctl->rounds, 4, cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaMemcpyAsync(v->h_rounds + 1, &s->d_ctl->wait_site, 4, cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaStreamSynchronize(st));
    v->steps++;
    if (v->h_rd->status == DS_TIMEOUT) {
        // the next step must find the ring empty
        cudaMemsetAsync(s->d_ring, 0xFF, ((u64)s->ring_mask + 1) * 8, st);
        cudaMemsetAsync(s->d_aq, 0, AQ_WORDS * 4, st);
        cudaStreamSynchronize(st);
        return set_error(PFG_ERR_DEVICE_TIMEOUT, "device-side wait timed out: %s made no progress for %llu ms",
                         wait_site_name(v->h_rounds[1]), (unsigned long long)(device_timeout_ns() / 1000000ull));
    }
    if (v->h_rd->status != DS_OK) return set_error(PFG_ERR_CUDA, "serving machine status %u", v->h_rd->status);

    // ---- retire finished slots ----
    const double t_done = v->now_us();
    u32 done = 0;
    for (u32 i = 0; i < S; ++i) {
        SlotInfo& sl = v->slots[i];
        if (!sl.used || v->h_done[i] == 0u) continue;
        pfg_query_result r;
        r.id = sl.req.id;
        r.src = sl.req.src;
        r.dst = sl.req.dst;
        r.dist = (u32)(v->h_out[i] >> 32);
        r.slot = i;
        r.submit_us = sl.req.submit_us;
        r.admit_us = sl.admit_us;
        r.finish_us = t_done;
        v->results.push_back(r);
        sl.used = false;
        ++done;
    }
    if (admitted_out) *admitted_out = m;
    if (completed_out) *completed_out = done;
    return PFG_OK;
}

extern "C" pfg_status pfg_server_results(pfg_server* v, pfg_query_result* out, uint32_t cap, uint32_t* n_out) {
    if (!v || !n_out || (cap && !out)) return set_error(PFG_ERR_INVALID_ARGUMENT, "bad argument");
    const u32 k = (u32)std::min<size_t>(cap, v->results.size());
    for (u32 i = 0; i < k; ++i) out[i] = v->results[i];
    v->results.erase(v->results.begin(), v->results.begin() + k);
    *n_out = k;
    return PFG_OK;
}

extern "C" uint32_t pfg_server_pending(const pfg_server* v) { return v ? (uint32_t)v->pending.size() : 0u; }
extern "C" uint32_t pfg_server_slots(const pfg_server* v) { return v ? v->S : 0u; }
extern "C" uint32_t pfg_server_in_flight(const pfg_server* v) {
    if (!v) return 0u;
    u32 k = 0;
    for (const auto& s : v->slots) k += s.used ? 1u : 0u;
    return k;
}
extern "C" double pfg_server_now_us(const pfg_server* v) { return v ? v->now_us() : 0.0; }
extern "C" pfg_solver* pfg_server_solver(pfg_server* v) { return v ? v->s : nullptr; }
