// pfg_common.cuh - device-side types and helpers of the B200 SSSP / A* engine.
//
// Layout in HBM (one solver):
//   adj    uint2[m_pad]   (col, w) pairs; every row starts on a 32-byte boundary
//                         (4 arcs) and is padded with (self, 0xFFFFFFFF) arcs, so a
//                         thread reads a whole row of a road graph in one sector
//                         with 128-bit loads. Rows keep the caller's order, which
//                         is sorted by weight (reference: src/graph.cpp:57-74), so
//                         the light arcs (w <= Delta) of a row are a prefix.
//   prow   u32[n+1]       padded row starts (multiples of 4).
//   x, y   f64[n]         coordinates for the A* heuristic (optional).
//   state  u64[K*n]       packed (dist << 32) | parent; one atomicMin updates both
//                         and an equal distance keeps the smaller parent
//                         (reference: src/gpu_kernels.cuh:11-13, 96-121).
//   queues u32[K*n] x 5   near ping-pong, far ping-pong, R (heavy set).
//   stamps u32[K*n] x 3   dedup words for near / far / R: an item is queued for
//                         epoch E iff stamp == E. Epochs only grow, so nothing is
//                         cleared between rounds or runs (the reference clears a
//                         bitmask bit per item, src/gpu_kernels.cuh:124-132).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pfg {

typedef uint32_t u32;
typedef uint64_t u64;

constexpr u32 INF32 = 0xFFFFFFFFu;
constexpr u32 NO_PARENT = 0xFFFFFFFFu;
constexpr u64 STATE_INIT = 0xFFFFFFFFFFFFFFFFull;  // (INF << 32) | NO_PARENT
constexpr u32 PAD_W = 0xFFFFFFFFu;                 // weight of a padding arc
constexpr u32 ROW_ALIGN = 4;                       // arcs per 32-byte sector

// Phases of the persistent kernel's state machine.
enum Phase : u32 {
    PH_INIT = 0,   // state initialisation (grid-stride), then seeding
    PH_LIGHT = 1,  // relax light arcs of the near queue
    PH_SCAN = 2,   // bucket start: relax far items inside the new window, keep the rest
    PH_HEAVY = 3,  // relax heavy arcs of the bucket's settled set R
    PH_NAIVE = 4,  // Bellman-Ford sweep over all vertices (naive mode)
    PH_COMPACT = 5,// prefix-sum compaction of the flagged next frontier
    PH_DONE = 6,
    PH_PAUSE = 7,  // serving: the step's round budget is spent; Ctl::resume_phase is next
    PH_ASYNC = 8   // bucket drained without rounds: CTAs pull work from the ring queue
};

// Ring queue of the asynchronous bucket phase: counters in RunParams::aq, one
// 128-byte line each (u32 index).
enum RingCounter : u32 { AQ_HEAD = 0, AQ_TAIL = 32, AQ_DONE = 64, AQ_BUSY = 96, AQ_IDLE = 128, AQ_HUBS = 160,
                         AQ_BEAT = 192, AQ_WORDS = 224 };
// AQ_BEAT: heartbeat, bumped by every working pass of an asynchronous drain. A
// CTA that waits (for work, or at the barrier after leaving a drain) measures its
// time limit from the last change of the heartbeat, so a long but progressing
// drain (one CTA walking a long chain) never reads as a hang.
// A ring entry is (distance the vertex was queued with) << 32 | state index;
// RING_FREE marks a free slot (no entry has index 2^32 - 1 and distance INF).
constexpr unsigned long long RING_FREE = ~0ull;

// Independent bucket windows (RunParams::iw): a ring entry whose index has
// IW_FAR_BIT set is an item of its instance's far pile, queued when the
// instance's window advanced; its high half is the start of that window.
constexpr u32 IW_FAR_BIT = 0x80000000u;
constexpr u32 IW_MAX_INST = 256;  // instances of one run that may use independent windows
enum IwMisc : u32 { IW_ACTIVE = 0, IW_MAXEP = 1, IW_ADVANCES = 2, IW_MISC_WORDS = 32 };
// Device words of the independent-window block for k instances: window words
// (u64 [k]), pending units [k], far-pile counts [2k], far-pile minima [2k],
// then IW_MISC_WORDS counters.
__host__ __device__ constexpr unsigned long long iw_words(unsigned k) { return 7ull * k + IW_MISC_WORDS + 2ull; }

// Grid tier of the hybrid mapping: an item whose selected arcs exceed
// RunParams::hub_min is published as a hub record, and any CTA claims chunks
// of hub_chunk arcs of it (aq[AQ_HUBS] counts the records of the current
// round / bucket drain; records are valid for the round descriptor's near
// epoch only, so nothing is cleared between rounds).
struct __align__(32) HubRec {
    u32 gi, eb, ee;  // state index of the item, its selected arc range
    u32 ready;       // near epoch of the round that published it (fields visible)
    u32 next;        // next unclaimed arc offset (atomicAdd by hub_chunk)
    u32 done;        // arcs relaxed (asynchronous buckets: the last chunk ends the record's busy unit)
    u32 pad0, pad1;
};

// Run modes (reference GpuAlgo, include/gpu_sssp.h:10-14).
enum RunMode : int { MODE_NAIVE = 0, MODE_FRONTIER = 1, MODE_DELTA = 2 };

// Queue counter slots in Ctl::cnt.
enum CounterSlot : u32 { C_NEAR0 = 0, C_NEAR1 = 1, C_FAR0 = 2, C_FAR1 = 3, C_R = 4, C_COUNT = 8 };

// Device status words (match pfg_status values).
enum DevStatus : u32 { DS_OK = 0, DS_BAD_SOURCE = 1, DS_BAD_GRAPH = 2, DS_NOT_CONVERGED = 4, DS_TIMEOUT = 5 };

// Which device-side wait ran out of time (Ctl::wait_site; outside the words a
// transition stores back, so a concurrent transition never erases it).
enum WaitSite : u32 { WS_NONE = 0, WS_RING_PUSH = 1, WS_DRAIN_IDLE = 2, WS_SPILL_SLOT = 3, WS_RING_SLOT = 4,
                      WS_BARRIER = 5, WS_LOCAL_SLOT = 6 };
inline const char* wait_site_name(u32 w) {
    switch (w) {
        case WS_RING_PUSH: return "a ring-queue push waiting for a free slot";
        case WS_DRAIN_IDLE: return "an idle CTA of an asynchronous bucket waiting for work";
        case WS_SPILL_SLOT: return "a claimed-list spill waiting for a free ring slot";
        case WS_RING_SLOT: return "a ring-queue pop waiting for its item to be written";
        case WS_BARRIER: return "the grid barrier";
        case WS_LOCAL_SLOT: return "a CTA work-queue slot hand-over";
    }
    return "a device-side wait";
}

// Round descriptor: everything a CTA needs to run the next round. Written by
// the transition, read by every CTA with five 16-byte loads after a barrier.
struct __align__(16) Rd {
    u32 phase, in_count, in_buf, far_in;   // input of the round
    u32 far_out, status, delta, heavy;     // far pile receiving pushes, Delta of the bucket
    u32 near_epoch, far_epoch, r_epoch, naive_in;  // dedup stamps of this round's outputs
    u32 flag_epoch, map_mode;
    u32 async_bkt;                         // 1: this bucket is drained asynchronously (ring + claimed lists)
    u32 in_kind;                           // ASYNC input slice: 0 far pile, 1 near queue (the seeds)
    u64 lo, hi;                            // bucket window [lo, hi) on the key
};

// Control block in device memory (16-byte aligned, a multiple of 16 bytes so
// the CTA running a transition loads and stores it with vector accesses).
// The host rewrites everything before `persist` before each run; the epoch
// counters after it carry over from run to run so stamp words never need
// clearing.
struct __align__(16) Ctl {
    u32 bar_count;     // barrier tickets taken in this run (grows by gridDim.x per barrier)
    u32 bar_gen;       // barriers completed in this run
    u32 wait_site;     // WaitSite of the first wait that ran out of time (0: none)
    u32 pad_b1;
    Rd rd;
    u32 rounds;        // barrier epochs so far
    u32 iterations;    // rounds with a non-empty input
    u32 buckets;
    u32 round_cap;
    u32 delta0;        // Delta of the first bucket
    u32 changed;       // naive mode: some distance decreased this round
    u32 policy_calls;  // learned-policy decisions taken
    u32 bucket_near;   // items entering the current bucket (policy feature)
    u32 bucket_rounds; // rounds spent in the current bucket (policy feature)
    u32 step_left;     // serving: rounds left in this step
    u32 resume_phase;  // serving: phase to run when a paused machine resumes
    u32 pad_c2;
    u64 far_min[2];    // smallest key pushed to each far pile
    u32 cnt[C_COUNT];  // queue tails
    unsigned long long stats[4];  // edges, atomics, updates, pushes
    u64 bucket_edges;  // edges scanned up to the start of the bucket (policy feature)
    // edges scanned so far, flushed every round when the policy runs: one atomicAdd per CTA
    // into stripe (CTA index mod 16), so no single word takes thousands of atomics a round
    u64 edge_stripe[16];
    // --- persistent across runs ---
    u32 persist;       // marker: everything from here on survives between runs
    u32 near_epoch;    // last stamp used by near pushes
    u32 far_epoch;     // last stamp used by far pushes
    u32 r_epoch;       // last stamp used by R pushes
};
static_assert(sizeof(Ctl) % 16 == 0, "Ctl must be a multiple of 16 bytes");
static_assert(sizeof(Rd) == 80, "Rd layout");

// Learned Delta-policy network (3 hidden layers of 64, fp32).
constexpr int POL_IN = 12;
constexpr int POL_H = 64;
constexpr int POL_OUT = 16; // classes: schedule (c / 8: 0 async, 1 rounds) x Delta multiplier kPolicyMult[c % 8]
constexpr int TRACE_W = 16; // trace row: POL_IN features, then bucket index, Delta, items, rounds
struct PolicyNet {
    float w1[POL_H * POL_IN], b1[POL_H];
    float w2[POL_H * POL_H], b2[POL_H];
    float w3[POL_H * POL_H], b3[POL_H];
    float w4[POL_OUT * POL_H], b4[POL_OUT];
    float in_mean[POL_IN], in_scale[POL_IN];
};

// Parameters of one persistent run (passed by value as a __grid_constant__).
struct RunParams {
    const uint2* adj;
    const u32* prow;
    const double* x;
    const double* y;
    u32 n;
    u32 maxw;          // largest real arc weight
    double hscale;     // A* heuristic scale (0: h = 0)
    double avg_w, avg_deg;
    u32 m;
    u32 k;             // instances (sources); instance i owns [i*n, (i+1)*n)
    u32 total;         // k*n
    const u32* srcs;   // device [k]
    int astar;
    u32 target;
    double xt, yt;     // target coordinates (A*)
    int use_h;         // heuristic enabled
    u64* state;
    u32* nearq[2];
    u32* farq[2];
    u32* rq;
    u32* near_stamp;
    u32* far_stamp;
    u32* r_stamp;
    u32* naive_mask[2];// naive mode: activity bitmasks [ceil(n/32)]
    Ctl* ctl;
    u32 delta;         // Delta of the first bucket (fixed-Delta mode: all buckets)
    int mode;          // RunMode
    int prefix_scan;   // 1: flag + scan compaction instead of queue pushes
    int policy;        // 1: learned Delta policy picks each bucket's Delta
    float* trace;      // optional: TRACE_W floats per bucket advance (policy features)
    u32 trace_cap;     // rows available in trace
    // Uneven instances (batch API): instance i owns state words
    // [inst_off[i], inst_off[i+1]) and its graph's padded row starts begin at
    // prow[inst_rowbase[i]]. nullptr: uniform instances of one graph, i*n + v.
    const u32* inst_off;
    const u32* inst_rowbase;
    // Serving (continuous batching of A* queries on uniform slots i*n + v):
    // slot i searches from its source to inst_target[i]; its keys are
    // dist + h_i(v) + inst_phi[i], so a query admitted later enters the shared
    // bucket sequence at the current window. inst_far_cnt[i] counts the slot's
    // items in the far pile of the current bucket; a slot with none left at a
    // bucket advance is finished (inst_done[i] = round + 1).
    const u32* inst_target;
    const double* inst_tx;
    const double* inst_ty;
    const long long* inst_phi;
    u32* inst_far_cnt;
    u32* inst_active;
    u32* inst_done;
    u32 step_rounds;   // > 0: pause after this many rounds (serving steps)
    int resume;        // 1: continue a paused state machine instead of starting a run
    u32 eager;         // hybrid mapping: eager sub-rounds per round (0 = off)
    u32 eager_max_items;  // ... only in rounds whose input has at most this many items
    const PolicyNet* net;
    u64 timeout_ns;    // bound on every device-side wait
    // Asynchronous buckets (ring != nullptr): inside a bucket, every improvement
    // of a vertex into the window queues an entry (state index, new distance) in
    // the improving CTA's claimed list or in a ring of ring_mask + 1 slots
    // (RING_FREE when free), and any CTA pulls ring entries as soon as they are
    // written; the grid barrier runs once per bucket instead of once per
    // relaxation round.
    unsigned long long* ring;
    u32 ring_mask;
    // ROW_ALIGN when every row of the graph(s) occupies exactly ROW_ALIGN slots
    // (no row has more arcs): row u of a graph starts at prow[first row] +
    // ROW_ALIGN * u, so an item's arcs are addressed without loading prow.
    u32 row_stride;
    u32 short_rows;    // 1 when no row has more than 32 arcs: the CTA-cooperative path is never needed
    u32* aq;           // ring counters, see RingCounter
    int test_absent_cta;  // test hook: CTA 0 leaves at once, so every barrier wait runs out
    HubRec* hubs;      // hub records (nullptr: no row of the graph is long enough)
    u32 hub_cap;       // records available
    u32 hub_min;       // items with more selected arcs are published as hubs
    u32 hub_chunk;     // arcs per claimed chunk
    // Asynchronous drains by warp workers (warp_drain = 1, PFG_SCHEDULE_WARP): every warp of a CTA
    // takes entries from the CTA's shared-memory work queue on its own, with no
    // block barrier between batches; rows above hub_min_warp selected arcs are
    // worked in chunks by all warps of the CTA (and rows above hub_min by any
    // CTA through hub records, claimed hub_chunk_warp arcs at a time).
    // warp_drain = 0: the CTA works its claimed list in block-synchronous passes.
    u32 warp_drain;
    u32 hub_min_warp;
    u32 hub_chunk_warp;
    // Block-synchronous drain: claimed-list entries a CTA keeps beyond its pass
    // before it spills the rest to the ring while no CTA is idle (0: half a block).
    u32 spill_keep;
    u32 idle_ns;       // block-synchronous drain: longest idle poll interval (ns; 0: 64)
    // 1: entries of asynchronous buckets are relaxed with the distance they carry, without
    // reading the state first (about a third of the entries are stale and relaxed anyway;
    // set for single-source runs on graphs of short rows, which are latency-bound)
    u32 trust_entries;
    // Independent bucket windows (iw = 1; multi-source Delta-stepping on graphs without hub
    // rows and with every arc light): instance i advances its own window [lo, hi) as soon as
    // its own entries are drained, so no grid barrier separates buckets and CTAs whose
    // instance finished a bucket work on other instances' buckets instead of waiting for the
    // slowest one. iw_win[i] = hi << 32 | far epoch << 1 | far pile in use; iw_pend[i] counts
    // the instance's queued entries plus one unit per CTA holding some of them in shared
    // memory, so it is zero exactly when the instance's window is drained; its far piles are
    // farq[b] + i * n with iw_fcnt[b * k + i] items and smallest key iw_fmin[b * k + i].
    u32 iw;
    unsigned long long* iw_win;
    u32* iw_pend;
    u32* iw_fcnt;
    u32* iw_fmin;
    u32* iw_misc;
};

// ---------------------------------------------------------------------------
// Small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ u64 global_timer_ns() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// L2-coherent loads for data written by other CTAs during the same kernel.
__device__ __forceinline__ u64 ld_state(const u64* p) { return __ldcg(p); }
__device__ __forceinline__ u32 ld_cg(const u32* p) { return __ldcg(p); }
__device__ __forceinline__ u32 vload(const u32* p) { return *(const volatile u32*)p; }
__device__ __forceinline__ u32 ld_relaxed(const u32* p) {
    u32 v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ u32 ld_acquire(const u32* p) {
    u32 v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ u64 vload64(const u64* p) { return *(const volatile u64*)p; }
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Records that the wait at `site` ran out of time (the first such wait names
// the site) and ends the run with DS_TIMEOUT.
__device__ __forceinline__ void flag_timeout(Ctl* c, u32 site) {
    atomicCAS(&c->wait_site, (u32)WS_NONE, site);
    atomicCAS(&c->rd.status, (u32)DS_OK, (u32)DS_TIMEOUT);
}

__device__ __forceinline__ u32 st_dist(u64 s) { return (u32)(s >> 32); }
__device__ __forceinline__ u64 pack_state(u32 d, u32 p) { return ((u64)d << 32) | (u64)p; }

// Admissible, consistent Euclidean heuristic. Same formula as the
// reference's heuristicValue (include/heuristic.h:19-25) so that A* keys and
// pruning follow the reference: h = floor(scale * |p(v) - p(t)| * (1 - 1e-9)),
// clamped to 4e9.
__host__ __device__ __forceinline__ u32 heuristic_value(double xv, double yv, double xt,
                                                        double yt, double scale) {
    const double dx = xv - xt, dy = yv - yt;
    const double e = sqrt(dx * dx + dy * dy) * scale * (1.0 - 1e-9);
    if (!(e > 0.0)) return 0u;
    if (e >= 4.0e9) return 4000000000u;
    return (u32)e;
}

// 64-bit update of the packed state. Returns true when the distance strictly
// decreased (the caller then queues the vertex). An equal distance with a
// smaller parent wins the atomicMin but returns false, as in the reference
// (src/gpu_kernels.cuh:96-121).
//   AM 0: read-before-atomic + atomicMin   (reference MinRBA)
//   AM 1: read-before-atomic + CAS loop    (reference CasRBA)
//   AM 2: blind atomicMin                  (reference MinNoCheck)
template <int AM>
__device__ __forceinline__ bool relax_state(u64* addr, u32 nd, u32 parent, u32& atomics) {
    const u64 nv = pack_state(nd, parent);
    if constexpr (AM == 2) {
        atomics++;
        const u64 old = atomicMin((unsigned long long*)addr, (unsigned long long)nv);
        return st_dist(old) > nd;
    } else {
        u64 cur = ld_state(addr);
        if (cur <= nv) return false;
        if constexpr (AM == 0) {
            atomics++;
            const u64 old = atomicMin((unsigned long long*)addr, (unsigned long long)nv);
            return st_dist(old) > nd;
        } else {
            // Lock-free: every failed CAS means another thread lowered the word.
            while (true) {
                atomics++;
                const u64 old = atomicCAS((unsigned long long*)addr, (unsigned long long)cur,
                                          (unsigned long long)nv);
                if (old == cur) return st_dist(old) > nd;
                cur = old;
                if (cur <= nv) return false;
            }
        }
    }
}

// Claims item i for epoch e: true exactly once per (i, e). A single exchange
// (no read first): the stamp is almost never set already, and on the latency
// path one L2 round trip matters more than an occasional redundant atomic.
__device__ __forceinline__ bool claim_stamp(u32* stamp, u32 i, u32 e) {
    return atomicExch(stamp + i, e) != e;
}

// Warp-aggregated append: one atomicAdd per group of converged lanes.
__device__ __forceinline__ void queue_push(u32* q, u32* tail, u32 item) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    u32 base = 0;
    if (lane == leader) base = atomicAdd(tail, (u32)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    q[base + __popc(mask & ((1u << lane) - 1u))] = item;
}

// Warp-aggregated append to the ring queue. The slot of position i was freed
// by the consumer of position i - (ring_mask + 1); the compare-and-swap makes
// a writer that catches up with a slow consumer wait (bounded) instead of
// overwriting an unread item. Returns false if that wait timed out.
__device__ __forceinline__ bool ring_push(unsigned long long* ring, u32 mask_bits, u32* tail, unsigned long long item,
                                          u64 timeout_ns) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    u32 base = 0;
    if (lane == leader) base = atomicAdd(tail, (u32)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    unsigned long long* slot = ring + ((base + __popc(mask & ((1u << lane) - 1u))) & mask_bits);
    if (atomicCAS(slot, RING_FREE, item) == RING_FREE) return true;
    const u64 t0 = global_timer_ns();
    while (atomicCAS(slot, RING_FREE, item) != RING_FREE) {
        if (global_timer_ns() - t0 > timeout_ns) return false;
        __nanosleep(64);
    }
    return true;
}

}  // namespace pfg
