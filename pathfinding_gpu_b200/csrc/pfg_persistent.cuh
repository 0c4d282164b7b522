// pfg_persistent.cuh - device code of the persistent SSSP / A* kernel (included by
// pfg_persistent.cu, which is compiled once per instantiation group so that the
// kernel's instantiations build in parallel, and by pfg_kernels.cu for the
// shared-memory layout).
//
// One cooperative launch runs a whole SSSP / A* / multi-source query: the
// reference's host loops (runNaive / runFrontier / runDelta,
// src/gpu_sssp.cu:257-456) become a state machine inside one kernel, so no
// host round trip happens between relaxation rounds. Each round ends in a
// bounded grid barrier; the CTA that arrives last runs the transition (queue
// swaps, bucket advance, termination) while the others wait, and every CTA
// reads the new control block after the barrier.
//
// Round kinds (reference counterparts):
//   LIGHT  relax the light arcs (w <= Delta) of the near queue      relaxFrontierKernel<SEL_LIGHT / SEL_ALL>, src/gpu_kernels.cuh:207-288
//   SCAN   bucket advance fused with the first light round: far items inside
//          the new window are relaxed at once, the rest stay far  farMinKernel + farPartitionKernel, :386-436
//   HEAVY  relax the heavy arcs (w > Delta) of R                    relaxFrontierKernel<SEL_HEAVY>
//   NAIVE  Bellman-Ford sweep over all vertices with activity bits naiveRelaxKernel, :297-329
//   COMPACT prefix-sum compaction of flagged vertices               cub::DeviceScan + scatterKernel, :376-383
//
// The window of the next bucket comes from the smallest key pushed to the far
// pile (tracked per round with one atomicMin per CTA) instead of a separate
// farMin pass; that value is a lower bound of every live far key, so buckets
// are never skipped.
#pragma once
#include "pfg_common.cuh"
#include "pfg_kernels.h"

#include <atomic>
#include <cstddef>
#include <cstdio>

namespace pfg {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr u32 MAX_BS = 1024;
constexpr u32 COOP_MIN = 32;  // hybrid mapping: rows with >= 32 selected arcs are CTA-cooperative

enum Kind { K_LIGHT = 0, K_SCAN = 1, K_HEAVY = 2 };

// Multipliers of the automatic Delta that the learned policy chooses from
// (class c: multiplier kPolicyMult[c % 8], asynchronous bucket if c < 8).
static __constant__ float kPolicyMult[8] = {0.0625f, 0.125f, 0.25f, 0.5f, 1.f, 2.f, 4.f, 8.f};

// The round descriptor, copied to shared memory after every barrier.
typedef Rd Snap;

struct Local {
    u32 edges = 0, atomics = 0, updates = 0, pushes = 0;
    u32 edges_flushed = 0;  // value of `edges` at the last per-round flush (policy / trace)
    u32 spilled = 0;   // warp drain: this thread pushed to the ring since its warp's last batch ended
    u64 fmin = ~0ull;  // smallest key this thread pushed to the far pile this round
};

constexpr u32 CL_CAP = 2048;  // claimed-list entries per CTA (hybrid mapping)

// A row task of the warp drain. claim packs (generation:16 | len:24 | next:24):
// a chunk is claimed by a compare-and-swap that advances `next` while next < len,
// and a task cannot complete (and its slot be reused) while a claimed chunk is
// unfinished, so the fields read after a successful claim are the task's.
constexpr u32 TASK_CAP = 8;
struct __align__(16) RowTask {
    unsigned long long claim;
    unsigned long long ub;  // A* pruning bound of the item
    u32 gi, u, du, ib, inst, eb, len;
    u32 done;   // arcs relaxed; the chunk that completes the row closes the task
    u32 free;   // 1: the slot may take a new task
    u32 pad[3];
};
static_assert(sizeof(RowTask) == 64, "RowTask layout");

// Per-CTA shared memory of the hybrid mapping (dynamic shared memory). The
// edge-balanced mapping's per-thread arrays follow the struct, sized by the
// launch's block size (coop_bytes), so a small CTA keeps the rest of the
// SM's 228 KB as L1 for the arc, coordinate and row-offset loads.
struct Coop {
    u32 wsum[32];
    u32 cl[CL_CAP];  // near vertices claimed by this CTA (circular: position i is cl[i % CL_CAP])
    u32 cl_d[CL_CAP];  // asynchronous buckets: the distance each entry was queued with
    u32 cl_n;        // positions appended (may run past cl_head + CL_CAP; the excess went to a global queue)
    u32 cl_head;     // first position not yet taken (rounds: always 0; asynchronous buckets: advances)
    u32 cl_base;
    u32 pad;
    // Asynchronous drain by warp workers: cl and cl_d together hold the CTA's
    // work queue, CL_CAP 64-bit slots of (queued distance << 32 | state index),
    // RING_FREE when free. Positions are reserved with shared-memory atomics;
    // a slot is handed over by its contents (a pusher waits for RING_FREE, a
    // popper for an entry), so any warp pushes and any warp pops.
    u32 wq_head;     // positions reserved by poppers
    u32 wq_tail;     // positions reserved by pushers
    u32 wq_pending;  // work the CTA holds (see warp_drain); > 0 exactly while it holds a busy unit
    u32 wq_agent;    // 1 while one warp polls the ring / hub records / termination for the CTA
    u32 wq_exit;     // 1: the bucket is drained (or the run failed): every warp leaves
    u32 wq_idle;     // 1 while the CTA is counted in the ring's idle counter
    u32 wq_hint;     // idle CTAs last seen by this CTA: > 0 makes producers spill to the ring
    u32 wq_beats;    // batches relaxed by this CTA and global progress seen by its agent (wait limits)
    u32 wq_backoff;  // idle poll interval (ns), doubled while the agent finds nothing
    u32 hub_cursor;  // first hub record of the drain this CTA has not passed
    u32 wq_beat_seen;  // last value of the ring's heartbeat seen by the CTA's agent
    u32 task_open;   // row tasks posted and not yet complete
    u32 pad2[4];
    // Ring positions [lo, hi) the CTA's agent took from the ring (hi << 32 | lo);
    // any warp of the CTA pops batches from it.
    unsigned long long rr;
    unsigned long long pad3;
    // Row tasks: rows of more than RunParams::hub_min_warp selected arcs that a
    // warp met in its batch, worked in chunks by every warp of the CTA.
    RowTask task[TASK_CAP];
};
static_assert(sizeof(Coop) % 16 == 0, "the per-thread arrays after Coop need 16-byte alignment");
static_assert(offsetof(Coop, cl) % 8 == 0 && offsetof(Coop, cl_d) == offsetof(Coop, cl) + 4 * CL_CAP,
              "cl and cl_d form the 64-bit work-queue slots of the warp drain");
static_assert(offsetof(Coop, rr) % 8 == 0 && offsetof(Coop, task) % 16 == 0, "Coop alignment");
constexpr u32 WQ_CAP = CL_CAP;
constexpr u32 WQ_MASK = WQ_CAP - 1u;
__device__ __forceinline__ unsigned long long* wq_slots(Coop& cs) {
    return reinterpret_cast<unsigned long long*>(cs.cl);
}

// Bytes of dynamic shared memory for a CTA of `block` threads: Coop, then
// u64 ub[block], u32 off[block + 1], eb[block], u[block], du[block], ib[block], inst[block].
__host__ __device__ constexpr size_t coop_bytes(u32 block) { return sizeof(Coop) + (size_t)block * 32u + 4u; }

// Independent bucket windows (RunParams::iw): per-CTA arrays over the k
// instances, after the per-thread arrays: the window word of each instance the
// CTA holds, the entries of it the CTA holds (claimed list and the current
// pass), the entries of it finished in the current pass, the CTA's hold on it
// (IW_FREE / IW_HELD / IW_RELEASING), the instances whose windows the CTA
// advances next, and the holds its service warp releases during the next pass.
__host__ __device__ constexpr size_t iw_smem_offset(u32 block) { return (coop_bytes(block) + 15u) & ~(size_t)15u; }
__host__ __device__ constexpr size_t iw_smem_bytes(u32 k) { return (size_t)k * 28u + 16u; }
enum IwHold : u32 { IW_FREE = 0, IW_HELD = 1, IW_RELEASING = 2 };
struct IwSh {
    unsigned long long* win;
    u32 *lc, *fin, *held, *adv, *rel, *adv_n, *rel_n;
};
__device__ __forceinline__ IwSh iw_sh(const Coop* cs, u32 k) {
    unsigned char* b = (unsigned char*)cs + iw_smem_offset(blockDim.x);
    IwSh r;
    r.win = reinterpret_cast<unsigned long long*>(b);
    r.lc = reinterpret_cast<u32*>(b + 8u * k);
    r.fin = r.lc + k;
    r.held = r.fin + k;
    r.adv = r.held + k;
    r.rel = r.adv + k;
    r.adv_n = r.rel + k;
    r.rel_n = r.adv_n + 1;
    return r;
}

// ---------------------------------------------------------------------------
// Block-wide exclusive scan (warp shuffles + one pass over warp totals).
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 block_exclusive_scan(u32 v, u32* wsum, u32& total) {
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u32 nwarps = (blockDim.x + 31u) >> 5;
    u32 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(FULL, x, o);
        if (lane >= (u32)o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        u32 t = lane < nwarps ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(FULL, t, o);
            if (lane >= (u32)o) t += y;
        }
        if (lane < nwarps) wsum[lane] = t;  // inclusive prefix of warp totals
    }
    __syncthreads();
    total = wsum[nwarps - 1];
    const u32 warp_base = warp ? wsum[warp - 1] : 0u;
    __syncthreads();  // wsum may be reused right after
    return warp_base + x - v;
}

__device__ __forceinline__ u64 block_min_u64(u64 v, u64* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const u64 y = __shfl_down_sync(FULL, v, o);
        v = y < v ? y : v;
    }
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    u64 r = ~0ull;
    if (threadIdx.x == 0) {
        const u32 nwarps = (blockDim.x + 31u) >> 5;
        for (u32 i = 0; i < nwarps; ++i) r = red[i] < r ? red[i] : r;
    }
    return r;  // valid in thread 0
}

// ---------------------------------------------------------------------------
// Heuristic and light/heavy split
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 h_of(const RunParams& p, u32 v) {
    if (!p.use_h) return 0u;
    return heuristic_value(p.x[v], p.y[v], p.xt, p.yt, p.hscale);
}

// A* key of a vertex of instance `inst` at distance d: d + h(v) + phi, where the
// target (and so h) and the key offset phi are per instance when serving.
__device__ __forceinline__ u64 astar_key(const RunParams& p, u32 inst, u32 v, u64 d) {
    if (!p.use_h) return p.inst_phi ? (u64)((long long)d + __ldg(p.inst_phi + inst)) : d;
    if (p.inst_target) {
        const u32 h = heuristic_value(p.x[v], p.y[v], __ldg(p.inst_tx + inst), __ldg(p.inst_ty + inst), p.hscale);
        return (u64)((long long)d + (long long)h + __ldg(p.inst_phi + inst));
    }
    return d + heuristic_value(p.x[v], p.y[v], p.xt, p.yt, p.hscale);
}

// Pruning bound of an A* instance in key space: key(target) = dist(target) + phi
// (h(target) = 0), or "none" while the target is unreached.
__device__ __forceinline__ u64 astar_bound(const RunParams& p, u32 inst, u32 ib) {
    const u32 t = p.inst_target ? __ldg(p.inst_target + inst) : p.target;
    const u32 dt = st_dist(ld_state(p.state + ib + t));
    if (dt == INF32) return ~0ull;
    return p.inst_phi ? (u64)((long long)dt + __ldg(p.inst_phi + inst)) : (u64)dt;
}

// First arc of [r0, r1) whose weight exceeds delta (rows are sorted by weight).
__device__ __forceinline__ u32 light_end(const uint2* adj, u32 r0, u32 r1, u32 delta) {
    u32 lo = r0, hi = r1;
    while (lo < hi) {
        const u32 mid = lo + ((hi - lo) >> 1);
        if (__ldg(&adj[mid].y) <= delta) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Work queue of the warp drain (shared memory; any warp pushes, any warp pops)
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 vld_s(const u32* q) { return *(const volatile u32*)q; }

// Entries one warp takes at a time (one per lane).
constexpr u32 WQ_BATCH = 32;

// Reserves cnt push positions [base, base + cnt); false when the queue lacks
// room (or the reservation keeps losing races): the caller uses the ring.
__device__ __forceinline__ bool wq_reserve(Coop& cs, u32 cnt, u32& base) {
    u32 t = vld_s(&cs.wq_tail);
    for (int tries = 0; tries < 64; ++tries) {
        const u32 used = t - vld_s(&cs.wq_head);
        if ((int)used >= 0 && used + cnt > WQ_CAP) return false;
        const u32 o = atomicCAS(&cs.wq_tail, t, t + cnt);
        if (o == t) {
            base = t;
            return true;
        }
        t = o;
    }
    return false;
}

// Writes the entry of reserved position pos once the slot's previous entry has
// been taken (bounded wait; on timeout the run fails).
__device__ __forceinline__ void wq_write(Coop& cs, u32 pos, unsigned long long ent, const RunParams& p) {
    unsigned long long* slot = wq_slots(cs) + (pos & WQ_MASK);
    if (atomicCAS(slot, RING_FREE, ent) == RING_FREE) return;
    const u64 t0 = global_timer_ns();
    while (atomicCAS(slot, RING_FREE, ent) != RING_FREE) {
        if (global_timer_ns() - t0 > p.timeout_ns) {
            flag_timeout(p.ctl, WS_LOCAL_SLOT);
            return;
        }
        __nanosleep(20);
    }
}

// Warp-aggregated push of one entry per calling lane into the CTA's queue,
// counted as pending work first (the pushing warp holds pending work itself,
// so the count never reaches zero early). False for the whole group when the
// queue is full, or when other CTAs are idle and this CTA already keeps one
// entry per thread (a batch for each of its warps): the entries then go to
// the ring, where idle CTAs take them.
__device__ __forceinline__ bool wq_push(Coop& cs, unsigned long long ent, const RunParams& p) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    const u32 cnt = __popc(mask);
    u32 base = 0, ok = 0;
    if (lane == leader) {
        const u32 backlog = vld_s(&cs.wq_tail) - vld_s(&cs.wq_head);
        if (!(vld_s(&cs.wq_hint) > 0u && (int)backlog > (int)blockDim.x)) {
            atomicAdd(&cs.wq_pending, cnt);
            ok = wq_reserve(cs, cnt, base) ? 1u : 0u;
            if (!ok) atomicSub(&cs.wq_pending, cnt);
        }
    }
    ok = __shfl_sync(mask, ok, leader);
    if (!ok) return false;
    base = __shfl_sync(mask, base, leader);
    wq_write(cs, base + __popc(mask & ((1u << lane) - 1u)), ent, p);
    return true;
}

// ---------------------------------------------------------------------------
// Relaxation of one arc (u -> v, w) and queueing of the improved head.
// ---------------------------------------------------------------------------
// cl != nullptr (hybrid mapping): a claimed near vertex goes to the CTA's
// claimed list in shared memory, which is relaxed again in the same round
// (eager sub-rounds) and flushed to the global near queue at the end of the
// round; only overflow goes to the global queue directly.
// Appends gv, which this thread has just claimed (near: for the current
// window; else: for the far pile), to the claimed list, the ring, or a queue;
// nd is its new distance (carried by entries of asynchronous buckets).
// IW: independent windows (near entries only; cl is the CTA's Coop): the entry is
// counted as the CTA's, or gets a pending unit of its own when it overflows.
template <bool IW = false>
__device__ __forceinline__ void push_claimed(const RunParams& p, const Snap& s, u32 gv, u32 nd, bool near,
                                             u32 inst, Local& L, Coop* cl) {
    Ctl* c = p.ctl;
    L.pushes++;
    if constexpr (IW) {
        const u32 slot = atomicAdd(&cl->cl_n, 1u);
        if (slot - cl->cl_head < CL_CAP) {
            cl->cl[slot & (CL_CAP - 1u)] = gv;
            cl->cl_d[slot & (CL_CAP - 1u)] = nd;
            atomicAdd(iw_sh(cl, p.k).lc + inst, 1u);  // held by this CTA
            return;
        }
        atomicAdd(p.iw_pend + inst, 1u);  // counted before the entry can be taken
        __threadfence();
        if (!ring_push(p.ring, p.ring_mask, p.aq + AQ_TAIL, ((unsigned long long)nd << 32) | gv, p.timeout_ns))
            flag_timeout(c, WS_RING_PUSH);
        return;
    }
    if (!near) {
        queue_push(p.farq[s.far_out], &c->cnt[C_FAR0 + s.far_out], gv);
        if (p.inst_far_cnt) atomicAdd(p.inst_far_cnt + inst, 1u);
        return;
    }
    if (s.async_bkt && p.warp_drain) {
        // asynchronous bucket drained by warp workers: the CTA's work queue, else the ring
        const unsigned long long ent = ((unsigned long long)nd << 32) | gv;
        if (cl && wq_push(*cl, ent, p)) return;
        L.spilled = 1u;
        if (!ring_push(p.ring, p.ring_mask, p.aq + AQ_TAIL, ent, p.timeout_ns)) flag_timeout(c, WS_RING_PUSH);
        return;
    }
    if (cl) {
        const u32 slot = atomicAdd(&cl->cl_n, 1u);
        if (slot - cl->cl_head < CL_CAP) {
            cl->cl[slot & (CL_CAP - 1u)] = gv;
            cl->cl_d[slot & (CL_CAP - 1u)] = nd;
            return;
        }
    }
    if (s.async_bkt) {
        if (!ring_push(p.ring, p.ring_mask, p.aq + AQ_TAIL, ((unsigned long long)nd << 32) | gv, p.timeout_ns))
            flag_timeout(c, WS_RING_PUSH);
        return;
    }
    const u32 out = s.in_buf ^ 1u;
    queue_push(p.nearq[out], &c->cnt[C_NEAR0 + out], gv);
}

// Independent windows: gi (of instance inst) was improved to `key`, at or
// beyond its instance's window end. The far pile in use and its epoch come
// with the window word w; the pile's minimum is lowered for every such
// improvement, and the vertex is queued once per epoch (so a pile never holds
// more than n items).
__device__ __forceinline__ void iw_far_push(const RunParams& p, u32 gi, u32 inst, u32 key, u64 w, Local& L) {
    const u32 fs = (u32)w & 1u, fe = (u32)w >> 1;
    atomicMin(p.iw_fmin + fs * p.k + inst, key);
    if (claim_stamp(p.far_stamp, gi, fe)) {
        const u32 pos = atomicAdd(p.iw_fcnt + fs * p.k + inst, 1u);
        if (pos < p.n)
            p.farq[fs][(size_t)inst * p.n + pos] = gi;
        else  // (one push per vertex and epoch: cannot happen)
            atomicCAS(&p.ctl->rd.status, (u32)DS_OK, (u32)DS_NOT_CONVERGED);
        L.pushes++;
    }
}

// After gv's distance was lowered to a value of key `key`: flag it (prefix-scan
// compaction) or claim it for the window / the far pile and queue it. ub: the
// A* pruning bound; under independent windows (IW) the window word of the
// item's instance, whose high half is the window end.
template <bool ASTAR, bool IW = false>
__device__ __forceinline__ void after_improve(const RunParams& p, const Snap& s, u32 gv, u64 key, u32 nd,
                                              u32 inst, u64 ub, Local& L, Coop* cl) {
    L.updates++;
    if constexpr (IW) {
        if (key < (ub >> 32))
            push_claimed<true>(p, s, gv, nd, true, inst, L, cl);
        else
            iw_far_push(p, gv, inst, (u32)key, ub, L);
        return;
    }
    if (p.mode == MODE_NAIVE) {  // Bellman-Ford sweep: the head is active in the next sweep
        atomicOr(p.naive_mask[s.naive_in ^ 1u] + (gv >> 5), 1u << (gv & 31u));
        if (vload(&p.ctl->changed) == 0u) p.ctl->changed = 1u;
        return;
    }
    if (p.prefix_scan) {  // flag only; the COMPACT round builds the next frontier
        p.near_stamp[gv] = s.near_epoch;
        L.pushes++;
        return;
    }
    const bool near = key < s.hi;
    if (!near) L.fmin = key < L.fmin ? key : L.fmin;
    if (near && s.async_bkt) {
        // Asynchronous bucket: no claim. Every strict improvement queues an
        // entry with the distance it set; an entry whose vertex has been
        // improved again by the time it is taken is skipped (the later
        // improvement queued its own), so each value a vertex reaches in the
        // window is relaxed once, without a claim exchange on the push or a
        // release and fence on the take.
        push_claimed(p, s, gv, nd, true, inst, L, cl);
        return;
    }
    if (claim_stamp(near ? p.near_stamp : p.far_stamp, gv, near ? s.near_epoch : s.far_epoch))
        push_claimed(p, s, gv, nd, near, inst, L, cl);
}

// Candidate distance nd and key of arc (u -> v, w) from du; false for a
// padding arc, a distance that leaves 32 bits, or (A*) a pruned key.
template <bool ASTAR>
__device__ __forceinline__ bool arc_candidate(const RunParams& p, u32 du, u64 ub, u32 inst, u32 v, u32 w,
                                              Local& L, u64& nd, u64& key) {
    if (w == PAD_W) return false;
    L.edges++;
    nd = (u64)du + w;
    if (nd >= INF32) return false;
    key = nd;
    if constexpr (ASTAR) {
        key = astar_key(p, inst, v, nd);
        if (key >= ub) return false;  // f(v) >= dist[target]: cannot improve the answer
    }
    return true;
}

template <bool ASTAR, int AM, bool IW = false>
__device__ __forceinline__ void relax_arc(const RunParams& p, const Snap& s, u32 u, u32 du,
                                          u32 ib, u64 ub, u32 inst, u32 v, u32 w, Local& L, Coop* cl) {
    u64 nd = 0, key = 0;
    if (!arc_candidate<ASTAR>(p, du, ub, inst, v, w, L, nd, key)) return;
    const u32 gv = ib + v;
    if (!relax_state<AM>(p.state + gv, (u32)nd, u, L.atomics)) return;
    after_improve<ASTAR, IW>(p, s, gv, key, (u32)nd, inst, ub, L, cl);
}

// Two arcs of one lane relaxed together: both state updates are issued before
// either result is used, so their L2 round trips overlap (same outcome as two
// relax_arc calls in a row).
template <bool ASTAR, int AM, bool IW = false>
__device__ __forceinline__ void relax_arc_pair(const RunParams& p, const Snap& s, bool va, u32 ua, u32 dua,
                                               u32 iba, u64 uba, u32 insta, uint2 aa, bool vb, u32 ub2, u32 dub,
                                               u32 ibb, u64 ubb, u32 instb, uint2 ab, Local& L, Coop* cl) {
    u64 nda = 0, keya = 0, ndb = 0, keyb = 0;
    const bool ga = va && arc_candidate<ASTAR>(p, dua, uba, insta, aa.x, aa.y, L, nda, keya);
    const bool gb = vb && arc_candidate<ASTAR>(p, dub, ubb, instb, ab.x, ab.y, L, ndb, keyb);
    const u32 gva = iba + aa.x, gvb = ibb + ab.x;
    bool ia, ibt;
    if constexpr (AM == 1) {
        ia = ga && relax_state<1>(p.state + gva, (u32)nda, ua, L.atomics);
        ibt = gb && relax_state<1>(p.state + gvb, (u32)ndb, ub2, L.atomics);
    } else {
        const u64 nva = pack_state((u32)nda, ua), nvb = pack_state((u32)ndb, ub2);
        bool ta = ga, tb = gb;
        if constexpr (AM == 0) {  // read before atomic: both reads in flight, then both atomics
            const u64 ca = ga ? ld_state(p.state + gva) : 0ull;
            const u64 cb = gb ? ld_state(p.state + gvb) : 0ull;
            ta = ga && ca > nva;
            tb = gb && cb > nvb;
        }
        unsigned long long oa = ~0ull, ob = ~0ull;
        if (ta) oa = atomicMin((unsigned long long*)(p.state + gva), (unsigned long long)nva);
        if (tb) ob = atomicMin((unsigned long long*)(p.state + gvb), (unsigned long long)nvb);
        L.atomics += (ta ? 1u : 0u) + (tb ? 1u : 0u);
        ia = ta && st_dist(oa) > (u32)nda;
        ibt = tb && st_dist(ob) > (u32)ndb;
    }
    if (ia) after_improve<ASTAR, IW>(p, s, gva, keya, (u32)nda, insta, uba, L, cl);
    if (ibt) after_improve<ASTAR, IW>(p, s, gvb, keyb, (u32)ndb, instb, ubb, L, cl);
}

// Thread tier: one thread walks its own arcs [eb, ee) with 128-bit loads
// (two arcs per load; rows start on 32-byte boundaries).
template <bool ASTAR, int AM>
__device__ __forceinline__ void relax_range_thread(const RunParams& p, const Snap& s, u32 u, u32 du,
                                                   u32 ib, u64 ub, u32 inst, u32 eb, u32 ee, Local& L,
                                                   Coop* cl = nullptr) {
    const uint4* a4 = reinterpret_cast<const uint4*>(p.adj);
    for (u32 e = eb & ~1u; e < ee; e += 2) {
        const uint4 q = __ldg(a4 + (e >> 1));
        if (e >= eb) relax_arc<ASTAR, AM>(p, s, u, du, ib, ub, inst, q.x, q.y, L, cl);
        if (e + 1 < ee) relax_arc<ASTAR, AM>(p, s, u, du, ib, ub, inst, q.z, q.w, L, cl);
    }
}

// State updates of up to four arcs (u -> hv[j], hw[j]) of one lane, all issued
// before any result is used (one dependent round of L2 round trips). Only the
// 32-bit candidate distances stay live across the round; A* keys of the
// improved heads are recomputed (cheap next to the relaxations).
template <bool ASTAR, int AM>
__device__ __forceinline__ void relax4(const RunParams& p, const Snap& s, u32 u, u32 du, u32 ib, u64 ub, u32 inst,
                                       const u32 (&hv)[4], const u32 (&hw)[4], Local& L, Coop* cl) {
    u32 nd[4];
    bool go[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        u64 d = 0, k = 0;
        go[j] = arc_candidate<ASTAR>(p, du, ub, inst, hv[j], hw[j], L, d, k);
        nd[j] = (u32)d;
    }
    if constexpr (AM == 1) {
#pragma unroll
        for (int j = 0; j < 4; ++j) go[j] = go[j] && relax_state<1>(p.state + ib + hv[j], nd[j], u, L.atomics);
    } else {
        if constexpr (AM == 0) {  // read before atomic: all reads in flight, then the atomics
            u64 cur[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) cur[j] = go[j] ? ld_state(p.state + ib + hv[j]) : 0ull;
#pragma unroll
            for (int j = 0; j < 4; ++j) go[j] = go[j] && cur[j] > pack_state(nd[j], u);
        }
        unsigned long long old[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            old[j] = go[j] ? atomicMin((unsigned long long*)(p.state + ib + hv[j]),
                                       (unsigned long long)pack_state(nd[j], u))
                           : ~0ull;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            L.atomics += go[j] ? 1u : 0u;
            go[j] = go[j] && st_dist(old[j]) > nd[j];
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (go[j]) {
            u64 key = nd[j];
            if constexpr (ASTAR) key = astar_key(p, inst, hv[j], nd[j]);
            after_improve<ASTAR>(p, s, ib + hv[j], key, nd[j], inst, ub, L, cl);
        }
    }
}

// Instance, state base, row base and local vertex of state index gi.
__device__ __forceinline__ void decode_item(const RunParams& p, u32 gi, u32& inst, u32& ib, u32& rb, u32& u) {
    rb = 0;  // first padded row start of the item's graph
    if (p.inst_off) {
        // uneven instances: last instance whose offset is <= gi
        u32 lo = 0, hi = p.k - 1;
        while (lo < hi) {
            const u32 mid = (lo + hi + 1) >> 1;
            if (__ldg(p.inst_off + mid) <= gi) lo = mid; else hi = mid - 1;
        }
        inst = lo;
        ib = __ldg(p.inst_off + lo);
        rb = __ldg(p.inst_rowbase + lo);
    } else {
        inst = p.k > 1 ? gi / p.n : 0u;
        ib = inst * p.n;
    }
    u = gi - ib;
}

// Reads one input item (a state index) and decides what to relax: returns
// false when the item is stale, pruned, or (SCAN) outside the new window -
// items of a later bucket are carried to the next far pile here. On true,
// [eb, ee) is the arc range of the round kind (light prefix / heavy suffix).
// The row bounds are loaded together with the state word (one round trip),
// or passed in (pre) by a caller that loaded them earlier. An entry of an
// asynchronous bucket passes the distance it was queued with (want): it is
// stale, and skipped, if the vertex has been improved since.
template <bool ASTAR>
__device__ __forceinline__ bool take_item(const RunParams& p, const Snap& s, u32 gi, int kind,
                                          Local& L, u32& u, u32& ib, u32& du, u64& ub, u32& inst,
                                          u32& eb, u32& ee, bool pre = false, u32 pr0 = 0u, u32 pr1 = 0u,
                                          u32 want = INF32) {
    Ctl* c = p.ctl;
    u32 rb;
    decode_item(p, gi, inst, ib, rb, u);
    u32 r0, r1;
    if (pre) {
        r0 = pr0;
        r1 = pr1;
    } else if (p.row_stride) {
        // fixed-stride rows: the arc block is known now, so it is fetched into
        // L1 while the state word is read (the relaxation's loads then hit)
        r0 = (rb ? __ldg(p.prow + rb) : 0u) + ROW_ALIGN * u;
        r1 = r0 + ROW_ALIGN;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p.adj + r0));
    } else {
        r0 = __ldg(p.prow + rb + u);
        r1 = __ldg(p.prow + rb + u + 1);
    }
    if (want != INF32 && p.trust_entries) {
        // single-source runs on short rows: the entry's own distance, without the state
        // read - a hop is one round trip instead of two, and a stale entry (its vertex
        // improved since) only relaxes upper bounds that the newer entry's values override
        du = want;
    } else {
        du = st_dist(ld_state(p.state + gi));
        if (want != INF32 && du != want) return false;  // stale: the newer entry relaxes it
    }
    bool act = du != INF32;
    u64 key = du;
    if constexpr (ASTAR) {
        ub = astar_bound(p, inst, ib);
        if (act) {
            key = astar_key(p, inst, u, du);
            if (key >= ub) act = false;
        }
    }
    if (kind == K_SCAN && act) {
        if (key < s.lo) {
            act = false;  // settled in an earlier bucket (stale far entry)
        } else if (key >= s.hi) {
            act = false;  // belongs to a later bucket: keep it far
            if (claim_stamp(p.far_stamp, gi, s.far_epoch)) {
                queue_push(p.farq[s.far_out], &c->cnt[C_FAR0 + s.far_out], gi);
                L.pushes++;
                if (p.inst_far_cnt) atomicAdd(p.inst_far_cnt + inst, 1u);
            }
            L.fmin = key < L.fmin ? key : L.fmin;
        }
    }
    if (!act) return false;
    if (kind == K_HEAVY) {
        eb = light_end(p.adj, r0, r1, s.delta);
        ee = r1;
    } else {
        eb = r0;
        ee = s.heavy ? light_end(p.adj, r0, r1, s.delta) : r1;
        // R = vertices of this bucket that own real heavy arcs.
        if (s.heavy && ee < r1 && __ldg(&p.adj[ee].y) != PAD_W) {
            if (claim_stamp(p.r_stamp, gi, s.r_epoch)) {
                queue_push(p.rq, &c->cnt[C_R], gi);
                L.pushes++;
            }
        }
    }
    return ee > eb;
}

// Edge-balanced CTA mapping: the selected arcs of all items of a chunk are
// numbered with a block-wide scan and dealt out one per thread, so every arc
// of a road-graph vertex and every slice of a hub row is relaxed in parallel
// (one dependent chain per arc). Called by every thread of the CTA.
template <bool ASTAR, int AM, bool IW = false>
__device__ __forceinline__ void relax_chunk_edges(const RunParams& p, const Snap& s, bool act, u32 u,
                                                  u32 du, u32 ib, u64 ub, u32 inst, u32 eb, u32 ee,
                                                  Local& L, Coop& cs, Coop* cl) {
    const u32 BS = blockDim.x;
    u32 total = 0;
    const u32 sz = act ? ee - eb : 0u;
    const u32 off = block_exclusive_scan(sz, cs.wsum, total);
    if (total == 0) return;  // block-uniform
    u64* c_ub = reinterpret_cast<u64*>(&cs + 1);
    u32* c_off = reinterpret_cast<u32*>(c_ub + BS);
    u32* c_eb = c_off + BS + 1;
    u32* c_u = c_eb + BS;
    u32* c_du = c_u + BS;
    u32* c_ib = c_du + BS;
    u32* c_inst = c_ib + BS;
    c_off[threadIdx.x] = off;
    c_eb[threadIdx.x] = eb;
    c_u[threadIdx.x] = u;
    c_du[threadIdx.x] = du;
    c_ib[threadIdx.x] = ib;
    c_ub[threadIdx.x] = ub;
    c_inst[threadIdx.x] = inst;
    if (threadIdx.x == 0) c_off[BS] = total;
    __syncthreads();
    for (u32 j = threadIdx.x; j < total; j += BS) {
        // owner = last slot with off <= j (zero-size slots repeat offsets, the
        // last of them is the owner); fixed-trip search, no divergence
        u32 lo = 0;
#pragma unroll
        for (u32 step = MAX_BS / 2; step > 0; step >>= 1) {
            const u32 cand = lo + step;
            if (cand < BS && c_off[cand] <= j) lo = cand;
        }
        const u32 e = c_eb[lo] + (j - c_off[lo]);
        const uint2 a = __ldg(p.adj + e);
        relax_arc<ASTAR, AM, IW>(p, s, c_u[lo], c_du[lo], c_ib[lo], c_ub[lo], c_inst[lo], a.x, a.y, L, cl);
    }
    __syncthreads();
}

// Writes the CTA's claimed list to the global near queue (one atomicAdd per CTA).
__device__ __forceinline__ void flush_claimed(const RunParams& p, const Snap& s, Coop& cs) {
    __syncthreads();
    const u32 total = min(cs.cl_n, CL_CAP);
    if (total > 0) {  // block-uniform
        const u32 out = s.in_buf ^ 1u;
        if (threadIdx.x == 0) cs.cl_base = atomicAdd(&p.ctl->cnt[C_NEAR0 + out], total);
        __syncthreads();
        u32* q = p.nearq[out] + cs.cl_base;
        for (u32 i = threadIdx.x; i < total; i += blockDim.x) q[i] = cs.cl[i];
        __syncthreads();
    }
    if (threadIdx.x == 0) cs.cl_n = 0;
}

// ---------------------------------------------------------------------------
// One round over an input array of items (state indices).
// ---------------------------------------------------------------------------
// Position of this thread's item in a chunk of blockDim.x items: item i goes to
// lane i / W of warp i % W (W warps), so a partly filled chunk spreads over all
// warps instead of filling the first ones.
__device__ __forceinline__ u32 item_slot() {
    const u32 W = blockDim.x >> 5;
    return (threadIdx.x & 31u) * W + (threadIdx.x >> 5);
}

// Warp-balanced relaxation: each warp numbers the selected arcs of its own
// lanes' items with a shuffle scan and deals them out one per lane (owner found
// by a 5-step shuffle search), with no block barrier. Used when no item of the
// CTA has more than WARP_ROW_MAX selected arcs, so a warp never carries a hub.
constexpr u32 WARP_ROW_MAX = 32;
template <bool ASTAR, int AM, bool IW = false>
__device__ __forceinline__ void relax_items_warp(const RunParams& p, const Snap& s, bool act, u32 u, u32 du,
                                                 u32 ib, u64 ub, u32 inst, u32 eb, u32 ee, Local& L, Coop* cl) {
    const u32 lane = threadIdx.x & 31u;
    const u32 sz = act ? ee - eb : 0u;
    u32 x = sz;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(FULL, x, o);
        if (lane >= (u32)o) x += y;
    }
    const u32 total = __shfl_sync(FULL, x, 31);
    const u32 off = x - sz;
    u32 j0 = 0;
    // More than 32 arcs left: two per lane, relaxed together (one dependent
    // chain of loads and atomics instead of two in a row).
    while (j0 + 32u < total) {  // warp-uniform; j0 may pass total when it ends
        const u32 ja = j0 + lane, jb = ja + 32u;
        u32 loa = 0, lob = 0;
#pragma unroll
        for (u32 step = 16; step > 0; step >>= 1) {
            if (__shfl_sync(FULL, off, loa + step) <= ja) loa += step;
            if (__shfl_sync(FULL, off, lob + step) <= jb) lob += step;
        }
        const u32 au = __shfl_sync(FULL, u, loa), adu = __shfl_sync(FULL, du, loa);
        const u32 aib = __shfl_sync(FULL, ib, loa), ainst = __shfl_sync(FULL, inst, loa);
        const u32 aeb = __shfl_sync(FULL, eb, loa) + (ja - __shfl_sync(FULL, off, loa));
        const u32 bu = __shfl_sync(FULL, u, lob), bdu = __shfl_sync(FULL, du, lob);
        const u32 bib = __shfl_sync(FULL, ib, lob), binst = __shfl_sync(FULL, inst, lob);
        const u32 beb = __shfl_sync(FULL, eb, lob) + (jb - __shfl_sync(FULL, off, lob));
        u64 aub = ~0ull, bub = ~0ull;
        if constexpr (ASTAR || IW) {
            aub = __shfl_sync(FULL, ub, loa);
            bub = __shfl_sync(FULL, ub, lob);
        }
        const bool vb = jb < total;
        const uint2 aa = __ldg(p.adj + aeb);
        const uint2 ab = vb ? __ldg(p.adj + beb) : make_uint2(0u, PAD_W);
        relax_arc_pair<ASTAR, AM, IW>(p, s, true, au, adu, aib, aub, ainst, aa, vb, bu, bdu, bib, bub, binst, ab, L,
                                      cl);
        j0 += 64u;
    }
    for (; j0 < total; j0 += 32) {  // warp-uniform
        const u32 j = j0 + lane;
        // owner = last lane whose offset is <= j (empty items repeat offsets)
        u32 lo = 0;
#pragma unroll
        for (u32 step = 16; step > 0; step >>= 1) {
            const u32 cand = lo + step;
            if (__shfl_sync(FULL, off, cand) <= j) lo = cand;
        }
        const u32 wu = __shfl_sync(FULL, u, lo), wdu = __shfl_sync(FULL, du, lo);
        const u32 wib = __shfl_sync(FULL, ib, lo), winst = __shfl_sync(FULL, inst, lo);
        const u32 web = __shfl_sync(FULL, eb, lo), woff = __shfl_sync(FULL, off, lo);
        u64 wub = ~0ull;
        if constexpr (ASTAR || IW) wub = __shfl_sync(FULL, ub, lo);
        if (j < total) {
            const uint2 a = __ldg(p.adj + web + (j - woff));
            relax_arc<ASTAR, AM, IW>(p, s, wu, wdu, wib, wub, winst, a.x, a.y, L, cl);
        }
    }
}

// Relaxes the selected arcs of the items held by the CTA's threads (at most one
// item per thread) with the mapping MAP. Called by every thread of the CTA.
template <bool ASTAR, int AM, int MAP, bool IW = false>
__device__ __forceinline__ void relax_items(const RunParams& p, const Snap& s, bool act, u32 u, u32 du,
                                            u32 ib, u64 ub, u32 inst, u32 eb, u32 ee, Local& L, Coop& cs,
                                            Coop* cl, int kind) {
    if constexpr (MAP == 0) {  // thread per item
        if (act) relax_range_thread<ASTAR, AM>(p, s, u, du, ib, ub, inst, eb, ee, L, cl);
    } else if constexpr (MAP == 1) {  // warp per item
        const u32 lane = threadIdx.x & 31u;
        unsigned ballot = __ballot_sync(FULL, act);
        while (ballot) {
            const int leader = __ffs(ballot) - 1;
            ballot &= ballot - 1;
            const u32 wu = __shfl_sync(FULL, u, leader), wdu = __shfl_sync(FULL, du, leader);
            const u32 wib = __shfl_sync(FULL, ib, leader), winst = __shfl_sync(FULL, inst, leader);
            const u64 wub = __shfl_sync(FULL, ub, leader);
            const u32 web = __shfl_sync(FULL, eb, leader), wee = __shfl_sync(FULL, ee, leader);
            for (u32 e = web + lane; e < wee; e += 32) {
                const uint2 a = __ldg(p.adj + e);
                relax_arc<ASTAR, AM>(p, s, wu, wdu, wib, wub, winst, a.x, a.y, L, cl);
            }
        }
    } else {
        // short rows only: each warp balances its own items; else the CTA does
        // (no CTA vote when no row of the graph has more than 32 arcs)
        if (!p.short_rows && __syncthreads_or(act && ee - eb > WARP_ROW_MAX))
            relax_chunk_edges<ASTAR, AM, IW>(p, s, act, u, du, ib, ub, inst, eb, ee, L, cs, cl);
        else
            relax_items_warp<ASTAR, AM, IW>(p, s, act, u, du, ib, ub, inst, eb, ee, L, cl);
    }
}

// Publishes the hub row [eb, ee) of item gi and returns its record index, or
// ~0u if the record table is full (the caller then relaxes the row itself). In
// an asynchronous drain (phase ASYNC) the record holds a busy unit until its
// last chunk is relaxed; in a round every CTA works the round's records before
// the barrier.
__device__ __forceinline__ u32 hub_publish_at(const RunParams& p, const Snap& s, u32 gi, u32 eb, u32 ee) {
    const bool drain = s.phase == PH_ASYNC;
    if (drain) atomicAdd(p.aq + AQ_BUSY, 1u);
    const u32 k = atomicAdd(p.aq + AQ_HUBS, 1u);
    if (k >= p.hub_cap) {
        if (drain) atomicSub(p.aq + AQ_BUSY, 1u);
        return ~0u;
    }
    HubRec* r = p.hubs + k;
    r->gi = gi;
    r->eb = eb;
    r->ee = ee;
    r->next = 0u;
    r->done = 0u;
    __threadfence();
    atomicExch(&r->ready, s.near_epoch);
    return k;
}

// Publishes a hub record (see hub_publish_at); false if the table is full.
__device__ __forceinline__ bool hub_publish(const RunParams& p, const Snap& s, u32 gi, u32 eb, u32 ee) {
    return hub_publish_at(p, s, gi, eb, ee) != ~0u;
}

// Claims the next chunk of a published hub row (records from the CTA's cursor
// s_hub[0] on; records without a chunk left are passed for good) and relaxes it
// with the whole CTA. Returns false if no chunk could be claimed. On true,
// s_hub[1] is the record and [s_hub[3], s_hub[4]) the chunk. Called by every
// thread of the CTA.
template <bool ASTAR, int AM>
__device__ __forceinline__ bool hub_chunk(const RunParams& p, const Snap& s, Local& L, Coop* cl, u32* s_hub) {
    __shared__ u32 s_u, s_du, s_ib, s_inst;
    __shared__ u64 s_ub;
    if (threadIdx.x == 0) {
        u32 k = s_hub[0], found = 0;
        const u32 cnt = min(ld_relaxed(p.aq + AQ_HUBS), p.hub_cap);
        for (; k < cnt; ++k) {
            HubRec* r = p.hubs + k;
            if (ld_acquire(&r->ready) != s.near_epoch) continue;  // not (yet) published: its owner relaxes it
            const u32 eb = __ldcg(&r->eb), ee = __ldcg(&r->ee);
            const u32 off = atomicAdd(&r->next, p.hub_chunk);
            if (off < ee - eb) {
                found = 1u;
                const u32 gi = __ldcg(&r->gi);
                s_hub[1] = k;
                s_hub[3] = eb + off;
                s_hub[4] = min(ee, eb + off + p.hub_chunk);
                u32 inst, ib, rb, u;
                decode_item(p, gi, inst, ib, rb, u);
                s_u = u;
                s_ib = ib;
                s_inst = inst;
                s_du = st_dist(ld_state(p.state + gi));
                s_ub = ~0ull;
                if constexpr (ASTAR) s_ub = astar_bound(p, inst, ib);
                break;
            }
        }
        s_hub[0] = k;
        s_hub[5] = found;
    }
    __syncthreads();
    if (!s_hub[5]) return false;  // block-uniform
    const u32 u = s_u, du = s_du, ib = s_ib, inst = s_inst;
    const u64 ub = s_ub;
    for (u32 e = s_hub[3] + threadIdx.x; e < s_hub[4]; e += blockDim.x) {
        const uint2 a = __ldg(p.adj + e);
        relax_arc<ASTAR, AM>(p, s, u, du, ib, ub, inst, a.x, a.y, L, cl);
    }
    __syncthreads();  // every push of the chunk has been performed
    return true;
}

template <bool ASTAR, int AM, int MAP>
__device__ __forceinline__ void round_items(const RunParams& p, const Snap& s, const u32* in, u32 count, int kind,
                            Local& L, Coop& cs) {
    const u32 BS = blockDim.x;
    // Hybrid mapping keeps claimed near vertices in shared memory (see relax_arc).
    // A heavy round between asynchronous buckets sends them to the ring, which
    // the drain that follows it empties.
    Coop* cl = (MAP == 2 && !p.prefix_scan && !(s.async_bkt && kind == K_HEAVY)) ? &cs : nullptr;
    // Every CTA takes one contiguous slice of the input, so a small frontier is
    // spread over all SMs (one arc chain per thread) instead of a few CTAs.
    const u32 per = (count + gridDim.x - 1u) / gridDim.x;
    const u32 sbeg = min(count, blockIdx.x * per);
    const u32 send = min(count, sbeg + per);
    for (u32 base = sbeg; base < send; base += BS) {
        const u32 idx = base + item_slot();
        u32 u = 0, ib = 0, du = INF32, eb = 0, ee = 0, inst = 0;
        u64 ub = ~0ull;
        bool act = false;
        u32 gi = 0;
        if (idx < send) {
            gi = ld_cg(in + idx);
            act = take_item<ASTAR>(p, s, gi, kind, L, u, ib, du, ub, inst, eb, ee);
        }
        if constexpr (MAP == 2) {  // hub rows go to the grid tier
            if (act && p.hubs && ee - eb > p.hub_min && hub_publish(p, s, gi, eb, ee)) act = false;
        }
        relax_items<ASTAR, AM, MAP>(p, s, act, u, du, ib, ub, inst, eb, ee, L, cs, cl, kind);
    }
    if constexpr (MAP == 2) {
        if (p.hubs && s.phase != PH_ASYNC) {
            // rounds: chunks of every hub record of the round before the barrier
            // (a CTA that published a record relaxes what nobody else claimed)
            __shared__ u32 s_hub[8];
            if (threadIdx.x == 0) s_hub[0] = 0u;
            __syncthreads();
            while (hub_chunk<ASTAR, AM>(p, s, L, cl, s_hub)) {
            }
        }
    }
    if constexpr (MAP == 2) {
        if (cl && !s.async_bkt) {  // (asynchronous buckets drain the claimed list themselves)
            // Eager sub-rounds: the vertices this CTA claimed for the next round
            // (keys inside the bucket window) are relaxed again right away, so
            // the wavefront advances several hops per grid barrier. They stay in
            // the claimed list and reach the global near queue at the flush, so
            // whatever happens here, the next round still processes them.
            // Only latency-bound rounds (small inputs) propagate eagerly: on
            // large frontiers the extra relaxations cost more than the barriers
            // they save.
            if (kind != K_HEAVY && count <= p.eager_max_items) {
                u32 lo = 0;
                for (u32 sub = 0; sub < p.eager; ++sub) {
                    __syncthreads();
                    const u32 hi = min(cs.cl_n, CL_CAP);
                    __syncthreads();
                    if (hi <= lo) break;  // block-uniform
                    for (u32 base = lo; base < hi; base += BS) {
                        const u32 idx = base + item_slot();
                        u32 u = 0, ib = 0, du = INF32, eb = 0, ee = 0, inst = 0;
                        u64 ub = ~0ull;
                        bool act = false;
                        if (idx < hi)
                            act = take_item<ASTAR>(p, s, cs.cl[idx], K_LIGHT, L, u, ib, du, ub, inst, eb, ee);
                        relax_items<ASTAR, AM, MAP>(p, s, act, u, du, ib, ub, inst, eb, ee, L, cs, cl, K_LIGHT);
                    }
                    lo = hi;
                }
            }
            flush_claimed(p, s, cs);
        }
    }
}

// ---------------------------------------------------------------------------
// Asynchronous drain of a bucket (phase ASYNC). Each CTA works through its own
// claimed list first (the entries its relaxations queued, kept in shared
// memory, up to one block of items per pass), so a wavefront advances hop by
// hop without any global queue traffic. Work moves between CTAs through the
// ring: a CTA spills the newest part of its backlog there when other CTAs are
// idle (or the backlog exceeds half a block), and a CTA with an empty list
// reserves a chunk of ring positions with a compare-and-swap on the head.
//
// Termination: AQ_BUSY counts the CTAs that still scan their slice of the
// bucket input or hold claimed-list items; AQ_DONE counts ring items relaxed.
// A CTA with nothing to do leaves once busy == 0 and done == tail: then no CTA
// holds work and every item ever pushed has been relaxed, so nothing can be
// pushed any more. A CTA takes a busy unit before it counts the ring chunk that
// gave it claimed items as done, and returns it only after the pushes of its
// last pass were performed, so the test never passes while work exists.
//
// Entries carry the distance they were queued with; a popped entry whose
// vertex has a smaller distance by now is stale and skipped. Every strict
// improvement queues an entry, so the entry of the value a vertex keeps is
// always relaxed, whatever order the CTAs run in.
// ---------------------------------------------------------------------------
template <bool ASTAR, int AM, int MAP>
__device__ __forceinline__ void async_drain(const RunParams& p, const Snap& s, Local& L, Coop& cs, bool busy_held) {
    __shared__ u32 s_src, s_h, s_n, s_spill, s_spill_from, s_spill_base, s_busy, s_idle;
    __shared__ u32 s_hub[8];
    constexpr u32 CLM = CL_CAP - 1u;
    const u32 G = gridDim.x, BS = blockDim.x;
    u32* aq = p.aq;
    Ctl* c = p.ctl;
    if (threadIdx.x == 0) {
        s_busy = busy_held ? 1u : 0u;
        s_idle = 0u;
        s_hub[0] = 0u;
    }
    __syncthreads();  // (each pass ends with a barrier after its pushes)
    for (;;) {
        if (threadIdx.x == 0) {
            // appends past cl_head + CL_CAP went to the ring already
            u32 tail = cs.cl_n;
            if ((int)(tail - (cs.cl_head + CL_CAP)) > 0) tail = cs.cl_head + CL_CAP;
            cs.cl_n = tail;
            const u32 local = tail - cs.cl_head;
            u32 src = 0, h = 0, n = 0, spill = 0;
            if (p.hubs && min(ld_relaxed(aq + AQ_HUBS), p.hub_cap) > s_hub[0]) {
                src = 3u;  // chunks of hub rows first: they are the longest chains
                n = 1u;
            } else if (local > 0u) {
                src = 1u;
                h = cs.cl_head;
                // up to two entries per thread (SSSP on graphs of short rows): a backlog of more
                // than a block is worked in one pass (both state reads in flight) instead of two
                // (1000 x 1000 grid, 128 sources: 30.0 -> 22.6 ms). A* instantiations keep one
                // (their registers are fuller), and so do graphs with long rows, whose
                // CTA-cooperative passes would double in length (R-MAT-20: 1.96 -> 2.56 ms).
                const u32 cap = (ASTAR || !p.short_rows) ? BS : 2u * BS;
                n = local < cap ? local : cap;
                const u32 backlog = local - n;
                const u32 keep = p.spill_keep ? p.spill_keep : BS / 2u;
                if (backlog >= 32u && (s_idle > 0u || backlog > keep))
                    spill = s_idle > 0u ? backlog / 2u : backlog - keep;
                cs.cl_head = h + n;
            } else {
                if (s_busy) {  // the last pass's pushes were performed before the barrier above
                    atomicSub(aq + AQ_BUSY, 1u);
                    s_busy = 0u;
                }
                bool idle = false;
                u64 t0 = global_timer_ns();
                u32 beat = ld_relaxed(aq + AQ_BEAT);
                u32 nap = 32u;  // idle poll interval (ns), doubled up to p.idle_ns
                for (u32 spin = 1;; ++spin) {
                    if ((spin & 15u) == 0u) {
                        if (vload(&c->rd.status) != DS_OK) break;
                        const u64 now = global_timer_ns();
                        const u32 b = ld_relaxed(aq + AQ_BEAT);
                        if (b != beat) {  // another CTA made progress: the wait is not a hang
                            beat = b;
                            t0 = now;
                        } else if (now - t0 > p.timeout_ns) {
                            flag_timeout(c, WS_DRAIN_IDLE);
                            break;
                        }
                    }
                    // done, then busy, then tail: a chunk's consumer takes its busy unit
                    // before it counts the chunk done, so done == tail with busy == 0 read
                    // in this order means no CTA held work in between
                    const u32 done = ld_acquire(aq + AQ_DONE);
                    const u32 busy = ld_acquire(aq + AQ_BUSY);
                    const u32 t = ld_acquire(aq + AQ_TAIL);
                    const u32 hh = ld_relaxed(aq + AQ_HEAD);
                    if ((int)(t - hh) > 0) {
                        nap = 32u;
                        const u32 avail = t - hh;
                        u32 want = (avail + G - 1u) / G;
                        want = want < 32u ? 32u : want;
                        want = want > BS ? BS : want;
                        want = want > avail ? avail : want;
                        if (atomicCAS(aq + AQ_HEAD, hh, hh + want) == hh) {
                            src = 2u;
                            h = hh;
                            n = want;
                            break;
                        }
                        continue;  // another CTA took these positions first
                    }
                    if (p.hubs && min(ld_relaxed(aq + AQ_HUBS), p.hub_cap) > s_hub[0]) {
                        src = 3u;
                        n = 1u;
                        break;
                    }
                    if (busy == 0u && done == t) break;  // the bucket is drained
                    if (!idle) {
                        atomicAdd(aq + AQ_IDLE, 1u);
                        idle = true;
                    }
                    __nanosleep(nap);
                    nap = min(2u * nap, p.idle_ns ? p.idle_ns : 64u);
                }
                if (idle) atomicSub(aq + AQ_IDLE, 1u);
            }
            s_src = src;
            s_h = h;
            s_n = n;
            s_spill = spill;
            if (spill) {
                s_spill_from = tail - spill;
                s_spill_base = atomicAdd(aq + AQ_TAIL, spill);
            }
        }
        __syncthreads();
        const u32 src = s_src, h = s_h, n = s_n, spill = s_spill;
        if (n == 0u) break;  // block-uniform
        if (threadIdx.x == 0) atomicAdd(aq + AQ_BEAT, 1u);
        if (src == 3u) {
            if (hub_chunk<ASTAR, AM>(p, s, L, MAP == 2 ? &cs : nullptr, s_hub) && threadIdx.x == 0) {
                if (cs.cl_n != cs.cl_head && !s_busy) {
                    atomicAdd(aq + AQ_BUSY, 1u);
                    s_busy = 1u;
                    __threadfence();  // busy is raised before the record can end
                }
                HubRec* r = p.hubs + s_hub[1];
                const u32 d = s_hub[4] - s_hub[3];
                if (atomicAdd(&r->done, d) + d == __ldcg(&r->ee) - __ldcg(&r->eb)) atomicSub(aq + AQ_BUSY, 1u);
            }
            continue;
        }
        if (spill) {
            // the newest part of the backlog goes to the ring for idle CTAs
            const u32 from = s_spill_from, base = s_spill_base;
            for (u32 i = threadIdx.x; i < spill; i += BS) {
                unsigned long long* slot = p.ring + ((base + i) & p.ring_mask);
                const unsigned long long ent = ((unsigned long long)cs.cl_d[(from + i) & CLM] << 32) |
                                               cs.cl[(from + i) & CLM];
                if (atomicCAS(slot, RING_FREE, ent) != RING_FREE) {
                    const u64 t0 = global_timer_ns();
                    while (atomicCAS(slot, RING_FREE, ent) != RING_FREE) {
                        if (global_timer_ns() - t0 > p.timeout_ns) {
                            flag_timeout(c, WS_SPILL_SLOT);
                            break;
                        }
                        __nanosleep(64);
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) cs.cl_n = from;
            __syncthreads();
        }
        u32 u = 0, ib = 0, du = INF32, eb = 0, ee = 0, inst = 0;
        u64 ub = ~0ull;
        bool act = false;
        const u32 my = item_slot();
        if (my < n) {
            unsigned long long ent;
            if (src == 1u) {
                ent = ((unsigned long long)cs.cl_d[(h + my) & CLM] << 32) | cs.cl[(h + my) & CLM];
            } else {
                unsigned long long* slot = p.ring + ((h + my) & p.ring_mask);
                ent = ld_relaxed64(slot);
                if (ent == RING_FREE) {
                    // reserved by a producer that has not written it yet
                    const u64 t0 = global_timer_ns();
                    while ((ent = ld_relaxed64(slot)) == RING_FREE) {
                        if (global_timer_ns() - t0 > p.timeout_ns) {
                            flag_timeout(c, WS_RING_SLOT);
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                if (ent != RING_FREE) *slot = RING_FREE;
            }
            if (ent != RING_FREE) {
                const u32 gi = (u32)ent;
                act = take_item<ASTAR>(p, s, gi, K_LIGHT, L, u, ib, du, ub, inst, eb, ee, false, 0u, 0u,
                                       (u32)(ent >> 32));
                if (MAP == 2 && act && p.hubs && ee - eb > p.hub_min && hub_publish(p, s, gi, eb, ee)) act = false;
            }
        }
        // the second entry of this thread (claimed-list passes of more than a block)
        u32 u2 = 0, ib2 = 0, du2 = INF32, eb2 = 0, ee2 = 0, inst2 = 0;
        u64 ub2 = ~0ull;
        bool act2 = false;
        if (!ASTAR && src == 1u && my + BS < n) {  // (n > BS only for short rows)
            const u32 q = (h + my + BS) & CLM;
            const u32 gi2 = cs.cl[q];
            act2 = take_item<ASTAR>(p, s, gi2, K_LIGHT, L, u2, ib2, du2, ub2, inst2, eb2, ee2, false, 0u, 0u,
                                    cs.cl_d[q]);
            if (MAP == 2 && act2 && p.hubs && ee2 - eb2 > p.hub_min && hub_publish(p, s, gi2, eb2, ee2))
                act2 = false;
        }
        u32 idle_now = 0u;
        if (threadIdx.x == 0) idle_now = ld_relaxed(aq + AQ_IDLE);
        relax_items<ASTAR, AM, MAP>(p, s, act, u, du, ib, ub, inst, eb, ee, L, cs, MAP == 2 ? &cs : nullptr, K_LIGHT);
        if (!ASTAR && n > BS)  // block-uniform
            relax_items<ASTAR, AM, MAP>(p, s, act2, u2, du2, ib2, ub2, inst2, eb2, ee2, L, cs, MAP == 2 ? &cs : nullptr,
                                        K_LIGHT);
        __syncthreads();  // every push of the pass has been performed
        if (threadIdx.x == 0) {
            s_idle = idle_now;
            if (src == 2u) {
                if (cs.cl_n != cs.cl_head && !s_busy) {
                    atomicAdd(aq + AQ_BUSY, 1u);
                    s_busy = 1u;
                    __threadfence();  // busy is raised before the chunk counts as done
                }
                atomicAdd(aq + AQ_DONE, n);
            }
        }
    }
    if (threadIdx.x == 0) {
        cs.cl_n = 0u;
        cs.cl_head = 0u;
    }
}

// ---------------------------------------------------------------------------
// Independent bucket windows (RunParams::iw = 1): one drain for the whole run.
//
// Every instance i has its own window [lo_i, hi_i). An improvement below hi_i
// queues an entry (claimed list or ring) as in an asynchronous bucket; one at
// or beyond it goes to the instance's far pile. iw_pend[i] counts the
// instance's entries in the ring plus one unit per CTA holding entries of it in
// its claimed list or its current pass, so it reaches zero exactly when nothing
// of the window is left anywhere: the CTA that releases the last unit advances
// the window (the next aligned window above the pile's smallest key, as a
// bucket advance does) and queues the pile's items in the ring, marked with
// IW_FAR_BIT and the old window end, for any CTA to classify and relax. An
// instance whose far pile is empty at its advance is finished; the drain ends
// when every instance is.
//
// Pending units: a ring entry carries one; the first entry of an instance that
// a CTA takes while holding none of it turns that unit into the CTA's hold, the
// others give theirs back; an entry pushed to the claimed list is covered by
// the hold, one that overflows to the ring gets its own unit before it is
// written, and so do entries spilled to the ring, before any of them is
// written. A CTA whose pass leaves it with no entry of an instance marks its
// hold IW_RELEASING; its service warp (warp 0, which relaxes nothing) releases
// it during the next pass, after a fence, so the far pushes and state updates
// of the CTA's passes are visible to whoever advances the window, and the fence
// and the returning atomic stay off the other warps' path. A ring entry of the
// instance taken before that cancels the release instead (the hold goes on);
// one compare-and-swap on the hold word decides which of the two happens. A
// CTA about to wait for work releases its marked holds first.
//
// Results do not depend on the order: every strict improvement is relaxed (near
// entries) or kept (far pile) until its window comes, so the final state is the
// same unique fixed point as with a shared window.
// ---------------------------------------------------------------------------

// Per warp: arr[key] += delta for each lane with v, one atomic per distinct
// key (every lane of the warp calls it).
__device__ __forceinline__ void warp_add_keyed(u32* arr, u32 key, int delta, bool v) {
    const unsigned vm = __ballot_sync(FULL, v);
    if (!v) return;
    const unsigned m = __match_any_sync(vm, key);
    if ((threadIdx.x & 31u) == (u32)(__ffs(m) - 1)) atomicAdd(arr + key, (u32)(delta * __popc(m)));
}

// Ring entries taken by this pass become the CTA's (every lane of the warp calls
// it; v: this lane took a ring entry of instance inst, whose window word is w).
__device__ __forceinline__ void iw_take_ring(const RunParams& p, const IwSh& sh, u32 inst, u64 w, bool v) {
    const unsigned vm = __ballot_sync(FULL, v);
    if (!v) return;
    const unsigned m = __match_any_sync(vm, inst);
    if ((threadIdx.x & 31u) == (u32)(__ffs(m) - 1)) {
        const u32 cnt = __popc(m);
        u32 give = cnt;
        if (atomicAdd(sh.lc + inst, cnt) == 0u) {
            // the CTA held no entry of the instance: a hold being released goes on,
            // otherwise one of the entries' units becomes the CTA's hold
            if (atomicCAS(sh.held + inst, (u32)IW_RELEASING, (u32)IW_HELD) != (u32)IW_RELEASING) {
                sh.held[inst] = IW_HELD;
                sh.win[inst] = w;
                give = cnt - 1u;
            }
        }
        if (give) atomicSub(p.iw_pend + inst, give);
    }
}

// Releases the hold on instance j unless a ring take cancelled it; lists j for
// an advance when that was the instance's last unit. fenced: the caller issued
// the fence that makes the CTA's earlier writes visible first.
__device__ __forceinline__ void iw_release(const RunParams& p, const IwSh& sh, u32 j, u32 K, Ctl* c) {
    if (atomicCAS(sh.held + j, (u32)IW_RELEASING, (u32)IW_FREE) != (u32)IW_RELEASING) return;
    if (atomicSub(p.iw_pend + j, 1u) == 1u) {
        // (an instance is listed at most once: its count stays zero until its advance)
        const u32 a = atomicAdd(sh.adv_n, 1u);
        if (a < K)
            sh.adv[a] = j;
        else
            atomicCAS(&c->rd.status, (u32)DS_OK, (u32)DS_NOT_CONVERGED);
    }
}

// Classifies an entry of instance inst (state index gi, carried value cv, window
// word w, state word sw read with it): a near entry (cv = the distance it was
// queued with) is stale when the vertex has been improved since; a far-pile item
// (far, cv = the window start of the advance that queued it) is relaxed when its
// distance lies in [cv, window end), kept far beyond it, and dropped below it
// (its window relaxed that value already). On true, [eb, ee) are the vertex's
// arcs (every arc is light under independent windows).
__device__ __forceinline__ bool take_iw(const RunParams& p, u32 gi, u32 inst, bool far, u32 cv, u64 w, u64 sw,
                                        Local& L, u32& u, u32& ib, u32& du, u32& eb, u32& ee) {
    ib = inst * p.n;
    u = gi - ib;
    u32 r0, r1;
    if (p.row_stride) {
        r0 = ROW_ALIGN * u;
        r1 = r0 + ROW_ALIGN;
    } else {
        r0 = __ldg(p.prow + u);
        r1 = __ldg(p.prow + u + 1);
    }
    du = st_dist(sw);
    if (!far) {
        if (du != cv) return false;  // stale: the newer entry relaxes it
    } else {
        if (du == INF32 || du < cv) return false;
        if (du >= (u32)(w >> 32)) {
            iw_far_push(p, gi, inst, du, w, L);
            return false;
        }
    }
    eb = r0;
    ee = r1;
    return ee > eb;
}

// Advances the window of instance j, whose pending count this CTA brought to
// zero: nothing of its window is left, so its far pile is complete. Called by
// every thread of the CTA.
static __device__ __noinline__ void iw_advance(const RunParams& p, const Snap& s, u32 j) {
    __shared__ u32 s_c, s_base, s_lo, s_fs;
    if (threadIdx.x == 0) {
        __threadfence();  // the releases that led here, before the pile is read
        const u32 k = p.k;
        const unsigned long long w = ld_relaxed64(p.iw_win + j);
        const u32 fs = (u32)w & 1u, fe = (u32)w >> 1, lo = (u32)(w >> 32);
        const u32 c = ld_relaxed(p.iw_fcnt + fs * k + j);
        const u32 est = ld_relaxed(p.iw_fmin + fs * k + j);
        u32 cnt = 0u;
        if (c == 0u || est == INF32) {
            atomicSub(p.iw_misc + IW_ACTIVE, 1u);  // nothing left beyond the window: finished
        } else {
            const u64 d = s.delta ? s.delta : 1u;
            u64 hi = ((u64)est / d + 1ull) * d;  // aligned, as a fixed-Delta bucket advance
            if (hi > 0xFFFFFFFFull) hi = 0xFFFFFFFFull;
            const u32 nfs = fs ^ 1u, nfe = fe + 1u;
            p.iw_fcnt[nfs * k + j] = 0u;
            p.iw_fmin[nfs * k + j] = INF32;
            p.iw_win[j] = (hi << 32) | ((unsigned long long)nfe << 1) | nfs;
            atomicAdd(p.iw_pend + j, c);  // one unit per queued item
            atomicMax(p.iw_misc + IW_MAXEP, nfe);
            atomicAdd(p.iw_misc + IW_ADVANCES, 1u);
            __threadfence();  // the window and the pending count before any item can be taken
            s_base = atomicAdd(p.aq + AQ_TAIL, c);
            cnt = c;
        }
        s_c = cnt;
        s_lo = lo;
        s_fs = fs;
    }
    __syncthreads();
    const u32 c = s_c;
    if (c) {
        const u32* pile = p.farq[s_fs] + (size_t)j * p.n;
        const unsigned long long hw = (unsigned long long)s_lo << 32;
        const u32 base = s_base, BS = blockDim.x;
        constexpr int U = 4;  // items per thread in flight: all loads, then all swaps
        for (u32 i0 = 0; i0 < c; i0 += U * BS) {
            unsigned long long ent[U];
            bool ok[U];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const u32 i = i0 + q * BS + threadIdx.x;
                ent[q] = i < c ? hw | (unsigned long long)(__ldcg(pile + i) | IW_FAR_BIT) : RING_FREE;
            }
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const u32 i = i0 + q * BS + threadIdx.x;
                ok[q] = i >= c || atomicCAS(p.ring + ((base + i) & p.ring_mask), RING_FREE, ent[q]) == RING_FREE;
            }
#pragma unroll
            for (int q = 0; q < U; ++q) {
                if (ok[q]) continue;
                // the slot's previous entry is not taken yet (bounded wait)
                unsigned long long* slot = p.ring + ((base + i0 + q * BS + threadIdx.x) & p.ring_mask);
                const u64 t0 = global_timer_ns();
                while (atomicCAS(slot, RING_FREE, ent[q]) != RING_FREE) {
                    if (global_timer_ns() - t0 > p.timeout_ns) {
                        flag_timeout(p.ctl, WS_SPILL_SLOT);
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
    }
    __syncthreads();
}

// Starts a run under independent windows (transition thread, at INIT): every
// instance's first window [0, Delta), one pending unit each, the sources queued
// in the ring with distance 0.
static __device__ __noinline__ void enter_iw(const RunParams& p, Ctl& sc, Rd& r) {
    const u32 k = p.k;
    const u64 hi = r.delta ? (u64)r.delta : 1ull;
    const u32 fe = r.far_epoch;
    for (u32 i = 0; i < k; ++i) {
        p.iw_win[i] = (hi << 32) | ((unsigned long long)fe << 1);
        p.iw_pend[i] = 1u;
        p.iw_fcnt[i] = 0u;
        p.iw_fcnt[k + i] = 0u;
        p.iw_fmin[i] = INF32;
        p.iw_fmin[k + i] = INF32;
        p.ring[i & p.ring_mask] = (unsigned long long)(i * p.n + p.srcs[i]);
    }
    p.iw_misc[IW_ACTIVE] = k;
    p.iw_misc[IW_MAXEP] = fe;
    p.iw_misc[IW_ADVANCES] = k;
    p.aq[AQ_HEAD] = 0u;
    p.aq[AQ_TAIL] = k;
    p.aq[AQ_DONE] = 0u;
    p.aq[AQ_BUSY] = 0u;
    p.aq[AQ_IDLE] = 0u;
    sc.cnt[C_NEAR0] = 0u;
    sc.cnt[C_NEAR1] = 0u;
    r.in_count = 0u;
    r.in_kind = 0u;
    r.lo = 0ull;
    r.hi = ~0ull;  // the shared test passes every key; each instance's window decides
    r.async_bkt = 1u;
    r.phase = PH_ASYNC;
}

// Position of this thread's entry in a pass of the independent-window drain:
// warps 1..W-1 relax, warp 0 serves (its lanes take no entry).
__device__ __forceinline__ u32 iw_item_slot() {
    const u32 W = blockDim.x >> 5, warp = threadIdx.x >> 5;
    return warp == 0u ? ~0u : (threadIdx.x & 31u) * (W - 1u) + (warp - 1u);
}

template <int AM>
__device__ __forceinline__ void inst_drain(const RunParams& p, const Snap& s, Local& L, Coop& cs) {
    __shared__ u32 s_src, s_h, s_n, s_spill, s_spill_from, s_spill_base, s_idle, s_j, s_nrel;
    constexpr u32 CLM = CL_CAP - 1u;
    const u32 G = gridDim.x, BS = blockDim.x, K = p.k;
    const u32 RS = BS - 32u;  // entries per pass and thread row: the relaxing warps' lanes
    u32* aq = p.aq;
    Ctl* c = p.ctl;
    const IwSh sh = iw_sh(&cs, K);
    for (u32 i = threadIdx.x; i < K; i += BS) {
        sh.lc[i] = 0u;
        sh.fin[i] = 0u;
        sh.held[i] = IW_FREE;
    }
    if (threadIdx.x == 0) {
        *sh.adv_n = 0u;
        *sh.rel_n = 0u;
        s_idle = 0u;
        s_nrel = 0u;
    }
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) {
            u32 tail = cs.cl_n;
            if ((int)(tail - (cs.cl_head + CL_CAP)) > 0) tail = cs.cl_head + CL_CAP;
            cs.cl_n = tail;
            const u32 local = tail - cs.cl_head;
            u32 src = 0, h = 0, n = 0, spill = 0;
            if (local == 0u && *sh.adv_n == 0u && *sh.rel_n) {
                // about to wait for work: release the marked holds now (they may be the
                // last units of their windows)
                __threadfence();
                for (u32 q = 0; q < *sh.rel_n; ++q) iw_release(p, sh, sh.rel[q], K, c);
                *sh.rel_n = 0u;
            }
            s_nrel = *sh.rel_n;  // the service warp releases these during the pass
            *sh.rel_n = 0u;
            if (*sh.adv_n) {
                src = 4u;  // window advances first: they start the next bucket of an instance
                n = 1u;
                *sh.adv_n -= 1u;
                s_j = sh.adv[*sh.adv_n];
            } else if (local > 0u) {
                src = 1u;
                h = cs.cl_head;
                const u32 cap = p.short_rows ? 2u * RS : RS;
                n = local < cap ? local : cap;
                const u32 backlog = local - n;
                const u32 keep = p.spill_keep ? p.spill_keep : BS / 2u;
                if (backlog >= 32u && (s_idle > 0u || backlog > keep))
                    spill = s_idle > 0u ? backlog / 2u : backlog - keep;
                cs.cl_head = h + n;
            } else {
                bool idle = false;
                u64 t0 = global_timer_ns();
                u32 beat = ld_relaxed(aq + AQ_BEAT);
                u32 nap = 32u;
                for (u32 spin = 1;; ++spin) {
                    if ((spin & 15u) == 0u) {
                        if (vload(&c->rd.status) != DS_OK) break;
                        const u64 now = global_timer_ns();
                        const u32 b = ld_relaxed(aq + AQ_BEAT);
                        if (b != beat) {
                            beat = b;
                            t0 = now;
                        } else if (now - t0 > p.timeout_ns) {
                            flag_timeout(c, WS_DRAIN_IDLE);
                            break;
                        }
                    }
                    const u32 act = ld_acquire(p.iw_misc + IW_ACTIVE);
                    const u32 t = ld_acquire(aq + AQ_TAIL);
                    const u32 hh = ld_relaxed(aq + AQ_HEAD);
                    if ((int)(t - hh) > 0) {
                        nap = 32u;
                        const u32 avail = t - hh;
                        u32 want = (avail + G - 1u) / G;
                        want = want < 32u ? 32u : want;
                        want = want > RS ? RS : want;
                        want = want > avail ? avail : want;
                        if (atomicCAS(aq + AQ_HEAD, hh, hh + want) == hh) {
                            src = 2u;
                            h = hh;
                            n = want;
                            break;
                        }
                        continue;
                    }
                    if (act == 0u) break;  // every instance is finished
                    if (!idle) {
                        atomicAdd(aq + AQ_IDLE, 1u);
                        idle = true;
                    }
                    __nanosleep(nap);
                    nap = min(2u * nap, p.idle_ns ? p.idle_ns : 64u);
                }
                if (idle) atomicSub(aq + AQ_IDLE, 1u);
            }
            s_src = src;
            s_h = h;
            s_n = n;
            s_spill = spill;
            if (spill) {
                s_spill_from = tail - spill;
                s_spill_base = atomicAdd(aq + AQ_TAIL, spill);
            }
        }
        __syncthreads();
        const u32 src = s_src, h = s_h, n = s_n, spill = s_spill;
        if (n == 0u) break;  // block-uniform (no hold is marked: the wait above released them)
        if (threadIdx.x == 0) atomicAdd(aq + AQ_BEAT, 1u);
        if (src == 4u) {
            if (threadIdx.x < 32u) {  // the marked holds, before the advance's barriers
                if (s_nrel) __threadfence();
                for (u32 q = threadIdx.x; q < s_nrel; q += 32u) iw_release(p, sh, sh.rel[q], K, c);
            }
            iw_advance(p, s, s_j);
            continue;
        }
        if (spill) {
            // the newest part of the backlog goes to the ring: each entry gets a pending
            // unit of its own before any of them is written, and leaves the CTA's count
            const u32 from = s_spill_from, base = s_spill_base;
            for (u32 b0 = 0; b0 < spill; b0 += BS) {
                const u32 i = b0 + threadIdx.x;
                const bool v = i < spill;
                const u32 inst = v ? cs.cl[(from + i) & CLM] / p.n : 0u;
                warp_add_keyed(p.iw_pend, inst, 1, v);
                warp_add_keyed(sh.lc, inst, -1, v);
            }
            __threadfence();
            __syncthreads();
            for (u32 i = threadIdx.x; i < spill; i += BS) {
                unsigned long long* slot = p.ring + ((base + i) & p.ring_mask);
                const unsigned long long ent = ((unsigned long long)cs.cl_d[(from + i) & CLM] << 32) |
                                               cs.cl[(from + i) & CLM];
                if (atomicCAS(slot, RING_FREE, ent) != RING_FREE) {
                    const u64 t0 = global_timer_ns();
                    while (atomicCAS(slot, RING_FREE, ent) != RING_FREE) {
                        if (global_timer_ns() - t0 > p.timeout_ns) {
                            flag_timeout(c, WS_SPILL_SLOT);
                            break;
                        }
                        __nanosleep(64);
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) cs.cl_n = from;
            __syncthreads();
        }
        u32 u = 0, ib = 0, du = INF32, eb = 0, ee = 0, inst = 0;
        unsigned long long w = 0ull, sw = 0ull;
        bool act = false;
        const u32 my = iw_item_slot();
        unsigned long long ent = RING_FREE;
        if (my < n) {
            if (src == 1u) {
                ent = ((unsigned long long)cs.cl_d[(h + my) & CLM] << 32) | cs.cl[(h + my) & CLM];
            } else {
                unsigned long long* slot = p.ring + ((h + my) & p.ring_mask);
                ent = ld_relaxed64(slot);
                if (ent == RING_FREE) {
                    const u64 t0 = global_timer_ns();
                    while ((ent = ld_relaxed64(slot)) == RING_FREE) {
                        if (global_timer_ns() - t0 > p.timeout_ns) {
                            flag_timeout(c, WS_RING_SLOT);
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                if (ent != RING_FREE) *slot = RING_FREE;
            }
        }
        const u32 lw = (u32)ent;
        const u32 gi = lw & ~IW_FAR_BIT;
        const bool have = ent != RING_FREE && gi < p.total;
        if (ent != RING_FREE && !have) atomicCAS(&c->rd.status, (u32)DS_OK, (u32)DS_NOT_CONVERGED);  // (cannot happen)
        if (have) {
            inst = gi / p.n;
            sw = ld_state(p.state + gi);  // (issued together with the window word)
            if (p.row_stride) asm volatile("prefetch.global.L1 [%0];" ::"l"(p.adj + ROW_ALIGN * (gi - inst * p.n)));
            // claimed-list entries: the CTA holds the instance, its window is in shared memory
            w = src == 1u ? sh.win[inst] : ld_relaxed64(p.iw_win + inst);
        }
        iw_take_ring(p, sh, inst, w, have && src == 2u);
        warp_add_keyed(sh.fin, inst, 1, have);
        if (have) act = take_iw(p, gi, inst, (lw & IW_FAR_BIT) != 0u, (u32)(ent >> 32), w, sw, L, u, ib, du, eb, ee);
        // the second entry of this thread (claimed-list passes of more than a row of entries)
        u32 u2 = 0, ib2 = 0, du2 = INF32, eb2 = 0, ee2 = 0, inst2 = 0;
        unsigned long long w2 = 0ull;
        bool act2 = false;
        const bool have2 = src == 1u && my < RS && my + RS < n;
        if (have2) {
            const u32 q = (h + my + RS) & CLM;
            const u32 gi2 = cs.cl[q];
            inst2 = gi2 / p.n;
            w2 = sh.win[inst2];
            act2 = take_iw(p, gi2, inst2, false, cs.cl_d[q], w2, ld_state(p.state + gi2), L, u2, ib2, du2, eb2,
                           ee2);
        }
        warp_add_keyed(sh.fin, inst2, 1, have2);
        if (threadIdx.x < 32u) {
            // service warp: the holds marked at the end of the last pass
            if (threadIdx.x == 0) s_idle = ld_relaxed(aq + AQ_IDLE);
            const u32 nr = s_nrel;
            if (nr) __threadfence();  // the earlier passes' far pushes and state updates first
            for (u32 q = threadIdx.x; q < nr; q += 32u) iw_release(p, sh, sh.rel[q], K, c);
        }
        relax_items<false, AM, 2, true>(p, s, act, u, du, ib, w, inst, eb, ee, L, cs, &cs, K_LIGHT);
        if (n > RS)  // block-uniform
            relax_items<false, AM, 2, true>(p, s, act2, u2, du2, ib2, w2, inst2, eb2, ee2, L, cs, &cs, K_LIGHT);
        __syncthreads();  // every push of the pass has been performed
        if (threadIdx.x < 32u) {
            // entries finished; a hold the CTA no longer needs is marked for release
            for (u32 j = threadIdx.x; j < K; j += 32u) {
                const u32 f = sh.fin[j];
                const u32 l = sh.lc[j] - f;
                if (f) {
                    sh.fin[j] = 0u;
                    sh.lc[j] = l;
                }
                if (l == 0u && sh.held[j] == IW_HELD) {
                    sh.held[j] = IW_RELEASING;
                    sh.rel[atomicAdd(sh.rel_n, 1u)] = j;  // (each held instance at most once)
                }
            }
            __syncwarp();
        }
    }
    if (threadIdx.x == 0) {
        cs.cl_n = 0u;
        cs.cl_head = 0u;
    }
}

// ---------------------------------------------------------------------------
// Asynchronous drain by warp workers (RunParams::warp_drain = 1).
//
// Every warp of a CTA works on its own: it takes up to WQ_BATCH entries (one
// per lane) from the CTA's shared-memory work queue, relaxes them and pushes
// the improvements back into the same queue, with no block barrier between
// batches, so a warp waiting on the L2 round trips of its batch never holds
// up the others and the next hop of the wavefront starts as soon as its entry
// is queued. Sources of work, in order: chunks of the CTA's row tasks (rows of
// more than hub_min_warp selected arcs, worked by all warps of the CTA), the
// work queue, the CTA's ring range (ring positions its agent took, popped by
// any warp), and - when all are empty - one poll by the CTA's agent (one warp
// at a time): chunks of other CTAs' hub rows, a new ring range, and, when the
// CTA holds no work, the drain's termination.
//
// Termination. cs.wq_pending counts the work the CTA holds (queued entries,
// entries being relaxed, the unrelaxed part of its ring range, open row
// tasks and chunks being relaxed); the CTA holds one unit of the ring's busy
// counter exactly while it is non-zero (taken by the warp that raises it from
// zero, before that warp marks any ring item done; returned by the warp that
// brings it to zero, after its pushes). Hub records hold their own busy unit
// until their last chunk is relaxed. The agent of a CTA that holds nothing ends
// the drain when it reads, in this order, the ring's done count, busy == 0 and
// the tail equal to that done count: every ring item pushed by then was
// relaxed, and no CTA held work in between, so no work can appear any more.
// ---------------------------------------------------------------------------
constexpr u32 TASK_CHUNK = 128;  // arcs of a row task claimed at a time (4 per lane)

__device__ __forceinline__ unsigned long long vld64_s(const unsigned long long* q) {
    return *(const volatile unsigned long long*)q;
}
__device__ __forceinline__ u32 claim_next(unsigned long long w) { return (u32)(w & 0xFFFFFFull); }
__device__ __forceinline__ u32 claim_len(unsigned long long w) { return (u32)((w >> 24) & 0xFFFFFFull); }
__device__ __forceinline__ u32 claim_gen(unsigned long long w) { return (u32)(w >> 48); }

// Returns k units of the CTA's pending work; the warp that brings the count
// to zero returns the CTA's busy unit (after its pushes are visible). Lane 0.
__device__ __forceinline__ void pending_done(Coop& cs, u32* aq, u32 k) {
    if (atomicSub(&cs.wq_pending, k) == k) {
        __threadfence();
        atomicSub(aq + AQ_BUSY, 1u);
    }
}
// Adds k units; the warp that raises the count from zero takes a busy unit
// (visible before anything it marks done). Lane 0.
__device__ __forceinline__ void pending_take(Coop& cs, u32* aq, u32 k) {
    if (atomicAdd(&cs.wq_pending, k) == 0u) {
        atomicAdd(aq + AQ_BUSY, 1u);
        __threadfence();
    }
}

// Prepares the CTA's work queue, ring range and row tasks for a bucket. All threads.
__device__ __forceinline__ void wq_reset(Coop& cs) {
    unsigned long long* wq = wq_slots(cs);
    for (u32 i = threadIdx.x; i < WQ_CAP; i += blockDim.x) wq[i] = RING_FREE;
    if (threadIdx.x < TASK_CAP) {
        cs.task[threadIdx.x].claim = 0ull;  // generation 0, nothing to claim
        cs.task[threadIdx.x].free = 1u;
    }
    if (threadIdx.x == 0) {
        cs.wq_head = cs.wq_tail = cs.wq_pending = 0u;
        cs.wq_agent = cs.wq_exit = cs.wq_idle = cs.wq_hint = 0u;
        cs.wq_backoff = 0u;
        cs.hub_cursor = 0u;
        cs.task_open = 0u;
        cs.rr = 0ull;
    }
    __syncthreads();
}

// Reserves up to max_take queued positions [h, h + n). Lane 0.
__device__ __forceinline__ u32 wq_pop(Coop& cs, u32 max_take, u32& h) {
    h = vld_s(&cs.wq_head);
    for (int tries = 0; tries < 64; ++tries) {
        const int avail = (int)(vld_s(&cs.wq_tail) - h);
        if (avail <= 0) return 0u;
        const u32 take = min((u32)avail, max_take);
        const u32 o = atomicCAS(&cs.wq_head, h, h + take);
        if (o == h) return take;
        h = o;
    }
    return 0u;
}

// Pops up to max_take positions [h, h + n) of the CTA's ring range. Lane 0.
__device__ __forceinline__ u32 rr_pop(Coop& cs, u32 max_take, u32& h) {
    unsigned long long w = vld64_s(&cs.rr);
    for (int tries = 0; tries < 64; ++tries) {
        const u32 lo = (u32)w, hi = (u32)(w >> 32);
        const int avail = (int)(hi - lo);
        if (avail <= 0) return 0u;
        const u32 take = min((u32)avail, max_take);
        const unsigned long long o = atomicCAS(&cs.rr, w, ((unsigned long long)hi << 32) | (lo + take));
        if (o == w) {
            h = lo;
            return take;
        }
        w = o;
    }
    return 0u;
}

// Entry of reserved queue position pos (waits, bounded, for its pusher to
// write it) and frees the slot.
__device__ __forceinline__ unsigned long long wq_take(Coop& cs, u32 pos, const RunParams& p) {
    volatile unsigned long long* slot = wq_slots(cs) + (pos & WQ_MASK);
    unsigned long long v = *slot;
    if (v == RING_FREE) {
        const u64 t0 = global_timer_ns();
        while ((v = *slot) == RING_FREE) {
            if (global_timer_ns() - t0 > p.timeout_ns) {
                flag_timeout(p.ctl, WS_LOCAL_SLOT);
                return RING_FREE;
            }
            __nanosleep(20);
        }
    }
    *slot = RING_FREE;
    return v;
}

// Entry of reserved ring position pos (waits, bounded, for its producer) and frees the slot.
__device__ __forceinline__ unsigned long long ring_take(const RunParams& p, u32 pos) {
    unsigned long long* slot = p.ring + (pos & p.ring_mask);
    unsigned long long ent = ld_relaxed64(slot);
    if (ent == RING_FREE) {
        const u64 t0 = global_timer_ns();
        while ((ent = ld_relaxed64(slot)) == RING_FREE) {
            if (global_timer_ns() - t0 > p.timeout_ns) {
                flag_timeout(p.ctl, WS_RING_SLOT);
                return RING_FREE;
            }
            __nanosleep(32);
        }
    }
    *slot = RING_FREE;
    return ent;
}

// Posts the row [eb, eb + len) of the calling lane's item as a row task of the
// CTA; false if every task slot is taken. The calling warp holds pending work,
// so the task's own unit is added without a busy hand-over.
__device__ __forceinline__ bool task_post(Coop& cs, u32 gi, u32 u, u32 du, u32 ib, u32 inst, u64 ub, u32 eb,
                                          u32 len) {
    if (len >= (1u << 24) - TASK_CHUNK) return false;
    for (u32 i = 0; i < TASK_CAP; ++i) {
        RowTask& t = cs.task[i];
        if (vld_s(&t.free) == 0u || atomicCAS(&t.free, 1u, 0u) != 1u) continue;
        t.gi = gi;
        t.u = u;
        t.du = du;
        t.ib = ib;
        t.inst = inst;
        t.ub = ub;
        t.eb = eb;
        t.len = len;
        t.done = 0u;
        atomicAdd(&cs.wq_pending, 1u);
        atomicAdd(&cs.task_open, 1u);
        __threadfence_block();  // fields before the claim word
        const unsigned long long gen = (unsigned long long)((claim_gen(vld64_s(&t.claim)) + 1u) & 0xFFFFu);
        atomicExch(&t.claim, (gen << 48) | ((unsigned long long)len << 24));
        return true;
    }
    return false;
}

// Claims the next chunk [e0, e1) of an open row task; returns its slot or ~0u. Lane 0.
__device__ __forceinline__ u32 task_claim(Coop& cs, u32& e0, u32& e1) {
    for (u32 i = 0; i < TASK_CAP; ++i) {
        RowTask& t = cs.task[i];
        unsigned long long w = vld64_s(&t.claim);
        for (int tries = 0; tries < 8; ++tries) {
            const u32 nx = claim_next(w), len = claim_len(w);
            if (nx >= len) break;
            const unsigned long long o = atomicCAS(&t.claim, w, w + TASK_CHUNK);
            if (o == w) {  // the task cannot complete before this chunk: its fields are stable
                const u32 eb = vld_s(&t.eb);
                e0 = eb + nx;
                e1 = eb + min(len, nx + TASK_CHUNK);
                return i;
            }
            w = o;
        }
    }
    return ~0u;
}

// Relaxes arcs [e0, e1) of one item with the calling warp, four arcs per lane
// in flight (so 128 arcs cost one dependent round of state updates).
template <bool ASTAR, int AM>
__device__ __forceinline__ void warp_relax_span(const RunParams& p, const Snap& s, u32 u, u32 du, u32 ib, u64 ub,
                                                u32 inst, u32 e0, u32 e1, Local& L, Coop* cl) {
    const u32 lane = threadIdx.x & 31u;
    for (u32 base = e0; base < e1; base += 128u) {
        u32 hv[4], hw[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const u32 e = base + lane + 32u * (u32)j;
            uint2 a = make_uint2(0u, PAD_W);
            if (e < e1) a = __ldg(p.adj + e);
            hv[j] = a.x;
            hw[j] = a.y;
        }
        relax4<ASTAR, AM>(p, s, u, du, ib, ub, inst, hv, hw, L, cl);
    }
}

// A hub chunk is done: the record's busy unit ends with its last chunk
// (pushes of the chunk are visible first). Lane 0.
__device__ __forceinline__ void hub_chunk_done(const RunParams& p, u32 k, u32 arcs) {
    HubRec* r = p.hubs + k;
    __threadfence();
    if (atomicAdd(&r->done, arcs) + arcs == __ldcg(&r->ee) - __ldcg(&r->eb)) atomicSub(p.aq + AQ_BUSY, 1u);
}

// The calling warp works hub record k (just published by one of its lanes, for
// an item it holds) until no chunk is left; idle CTAs' agents claim chunks too.
template <bool ASTAR, int AM>
__device__ __forceinline__ void warp_own_hub(const RunParams& p, const Snap& s, u32 k, u32 u, u32 du, u32 ib, u64 ub,
                                             u32 inst, Local& L, Coop* cl) {
    const u32 lane = threadIdx.x & 31u;
    HubRec* r = p.hubs + k;
    const u32 eb = __ldcg(&r->eb), len = __ldcg(&r->ee) - eb;
    for (;;) {
        u32 off = 0;
        if (lane == 0) off = atomicAdd(&r->next, p.hub_chunk_warp);
        off = __shfl_sync(FULL, off, 0);
        if (off >= len) break;
        const u32 e1 = min(len, off + p.hub_chunk_warp);
        warp_relax_span<ASTAR, AM>(p, s, u, du, ib, ub, inst, eb + off, eb + e1, L, cl);
        __syncwarp();
        if (lane == 0) hub_chunk_done(p, k, e1 - off);
    }
}

enum WarpSrc : u32 { WSRC_NONE = 0, WSRC_LOCAL = 1, WSRC_RANGE = 2, WSRC_HUB = 3, WSRC_TASK = 4, WSRC_EXIT = 5 };

// One poll by the CTA's agent (lane 0 of a warp that found no work; at most one
// warp of the CTA polls at a time). Returns WSRC_HUB with arcs [e0, e1) of hub
// record h claimed (counted as pending work), WSRC_RANGE after it installed a
// new ring range (counted as pending and marked done in the ring), WSRC_EXIT
// when the bucket is drained or the run failed, WSRC_NONE otherwise.
static __device__ u32 drain_agent(const RunParams& p, const Snap& s, Coop& cs, u32& h, u32& e0, u32& e1) {
    if (atomicCAS(&cs.wq_agent, 0u, 1u) != 0u) return WSRC_NONE;
    u32* aq = p.aq;
    u32 res = WSRC_NONE;
    if (vload(&p.ctl->rd.status) != DS_OK) res = WSRC_EXIT;
    if (res == WSRC_NONE && p.hubs) {
        // chunks of published hub rows (records not yet ready are passed: their publisher works them)
        const u32 cnt = min(ld_relaxed(aq + AQ_HUBS), p.hub_cap);
        u32 k = cs.hub_cursor;
        for (; k < cnt; ++k) {
            HubRec* r = p.hubs + k;
            if (ld_acquire(&r->ready) != s.near_epoch) continue;
            const u32 eb = __ldcg(&r->eb), ee = __ldcg(&r->ee);
            if (__ldcg(&r->next) >= ee - eb) continue;  // no chunk left
            const u32 off = atomicAdd(&r->next, p.hub_chunk_warp);
            if (off < ee - eb) {
                h = k;
                e0 = eb + off;
                e1 = min(ee, e0 + p.hub_chunk_warp);
                res = WSRC_HUB;
                break;
            }
        }
        cs.hub_cursor = k;
        if (res == WSRC_HUB) pending_take(cs, aq, 1u);
    }
    if (res == WSRC_NONE && (int)((u32)(vld64_s(&cs.rr) >> 32) - (u32)vld64_s(&cs.rr)) <= 0) {
        // a new ring range for the CTA's warps: a fair share of the ring, 32 .. blockDim.x items
        const u32 t = ld_acquire(aq + AQ_TAIL);
        const u32 hh = ld_relaxed(aq + AQ_HEAD);
        const int avail = (int)(t - hh);
        if (avail > 0) {
            u32 want = ((u32)avail + gridDim.x - 1u) / gridDim.x;
            want = min(max(want, 32u), blockDim.x);
            want = min(want, (u32)avail);
            if (atomicCAS(aq + AQ_HEAD, hh, hh + want) == hh) {
                pending_take(cs, aq, want);  // busy unit before the items count as done
                atomicAdd(aq + AQ_DONE, want);
                atomicExch(&cs.rr, ((unsigned long long)(hh + want) << 32) | hh);
                res = WSRC_RANGE;
            }
        }
    }
    if (res == WSRC_RANGE || res == WSRC_HUB) {
        if (cs.wq_idle) {
            atomicSub(aq + AQ_IDLE, 1u);
            cs.wq_idle = 0u;
        }
        cs.wq_backoff = 0u;
    } else if (res == WSRC_NONE) {
        if (vld_s(&cs.wq_pending) == 0u) {
            if (!cs.wq_idle) {
                atomicAdd(aq + AQ_IDLE, 1u);
                cs.wq_idle = 1u;
            }
            // done, then busy, then tail (see above)
            const u32 d = ld_acquire(aq + AQ_DONE);
            const u32 b = ld_acquire(aq + AQ_BUSY);
            const u32 t = ld_acquire(aq + AQ_TAIL);
            if (b == 0u && d == t) res = WSRC_EXIT;
        }
        if (res == WSRC_NONE) {
            cs.wq_hint = ld_relaxed(aq + AQ_IDLE);
            const u32 beat = ld_relaxed(aq + AQ_BEAT);
            if (beat != cs.wq_beat_seen) {  // another CTA made progress: this CTA's waits are not a hang
                cs.wq_beat_seen = beat;
                atomicAdd(&cs.wq_beats, 1u);
            }
            cs.wq_backoff = min(max(2u * cs.wq_backoff, 32u), 512u);
        }
    }
    if (res == WSRC_EXIT) {
        cs.wq_exit = 1u;
        if (cs.wq_idle) {
            atomicSub(aq + AQ_IDLE, 1u);
            cs.wq_idle = 0u;
        }
    }
    __threadfence_block();
    atomicExch(&cs.wq_agent, 0u);
    return res;
}

template <bool ASTAR, int AM, int MAP>
__device__ __forceinline__ void warp_drain(const RunParams& p, const Snap& s, Local& L, Coop& cs, bool busy_held) {
    const u32 lane = threadIdx.x & 31u;
    u32* aq = p.aq;
    Ctl* c = p.ctl;
    __syncthreads();  // the bucket's scan (if any) has queued its entries
    if (threadIdx.x == 0) {
        cs.wq_beats = 0u;
        cs.wq_beat_seen = 0u;
        // the busy unit the transition gave this CTA for its scan stays only while the CTA holds work
        if (busy_held && vld_s(&cs.wq_pending) == 0u) {
            __threadfence();  // (ring pushes of the scan first)
            atomicSub(aq + AQ_BUSY, 1u);
        }
    }
    L.spilled = 0u;
    __syncthreads();
    // entries per batch: about 64 selected arcs (one round of paired state updates
    // over the warp's lanes), between 4 and WQ_BATCH items
    const u32 B = (u32)max(4.0, min((double)WQ_BATCH, 64.0 / max(1.0, p.avg_deg)));
    bool waiting = false;  // lane 0: the warp is in a wait that started at t0 with progress count `seen`
    u32 seen = 0u, polls = 0u;
    u64 t0 = 0ull;
    for (;;) {
        u32 src = WSRC_NONE, n = 0, h = 0, e0 = 0, e1 = 0, hint = ~0u;
        if (lane == 0) {
            if (vld_s(&cs.wq_exit)) {
                src = WSRC_EXIT;
            } else if (vld_s(&cs.task_open) && (h = task_claim(cs, e0, e1)) != ~0u) {
                src = WSRC_TASK;
                atomicAdd(&cs.wq_pending, 1u);  // (the open task holds a unit: never from zero)
            } else if ((n = wq_pop(cs, B, h)) != 0u) {
                src = WSRC_LOCAL;
            } else if ((n = rr_pop(cs, B, h)) != 0u) {
                src = WSRC_RANGE;
            } else {
                src = drain_agent(p, s, cs, h, e0, e1);
                if (src == WSRC_RANGE) {
                    n = rr_pop(cs, B, h);
                    if (n == 0u) src = WSRC_NONE;
                }
            }
            if (src == WSRC_NONE) {
                const u32 b = vld_s(&cs.wq_beats);
                const u64 now = global_timer_ns();
                if (!waiting || b != seen) {
                    waiting = true;
                    seen = b;
                    t0 = now;
                } else if (now - t0 > p.timeout_ns) {
                    flag_timeout(c, WS_DRAIN_IDLE);
                    cs.wq_exit = 1u;
                    src = WSRC_EXIT;
                }
                if (src == WSRC_NONE) __nanosleep(max(vld_s(&cs.wq_backoff), 96u));
            } else if (src != WSRC_EXIT) {
                waiting = false;
                if ((++polls & 15u) == 0u) hint = ld_relaxed(aq + AQ_IDLE);  // refresh the spill hint now and then
            }
        }
        src = __shfl_sync(FULL, src, 0);
        if (src == WSRC_EXIT) break;
        if (src == WSRC_NONE) continue;
        n = __shfl_sync(FULL, n, 0);
        h = __shfl_sync(FULL, h, 0);
        if (src == WSRC_HUB || src == WSRC_TASK) {
            e0 = __shfl_sync(FULL, e0, 0);
            e1 = __shfl_sync(FULL, e1, 0);
            u32 u, du, ib, inst;
            u64 ub = ~0ull;
            if (src == WSRC_TASK) {
                const RowTask& t = cs.task[h];
                u = t.u;
                du = t.du;
                ib = t.ib;
                inst = t.inst;
                if constexpr (ASTAR) ub = t.ub;
            } else {  // another CTA's hub row: the record's item from its state word
                const u32 gi = __ldcg(&p.hubs[h].gi);
                u32 rb;
                decode_item(p, gi, inst, ib, rb, u);
                du = st_dist(ld_state(p.state + gi));
                if constexpr (ASTAR) ub = astar_bound(p, inst, ib);
            }
            warp_relax_span<ASTAR, AM>(p, s, u, du, ib, ub, inst, e0, e1, L, &cs);
            const bool spilled = __any_sync(FULL, L.spilled != 0u);
            L.spilled = 0u;
            if (lane == 0) {
                if (src == WSRC_HUB) {
                    hub_chunk_done(p, h, e1 - e0);
                } else {
                    RowTask& t = cs.task[h];
                    if (spilled) __threadfence();
                    if (atomicAdd(&t.done, e1 - e0) + (e1 - e0) == t.len) {  // the row is complete
                        atomicSub(&cs.task_open, 1u);
                        __threadfence_block();
                        atomicExch(&t.free, 1u);
                        pending_done(cs, aq, 1u);  // the task's unit
                    }
                }
                pending_done(cs, aq, 1u);  // the chunk's unit
                if ((atomicAdd(&cs.wq_beats, 1u) & 7u) == 0u) atomicAdd(aq + AQ_BEAT, 1u);
            }
            continue;
        }
        // a batch of entries, one per lane
        unsigned long long ent = RING_FREE;
        if (lane < n) ent = src == WSRC_LOCAL ? wq_take(cs, h + lane, p) : ring_take(p, h + lane);
        u32 u = 0, ib = 0, du = INF32, eb = 0, ee = 0, inst = 0, rec = ~0u;
        u64 ub = ~0ull;
        bool act = false;
        if (ent != RING_FREE) {
            const u32 gi = (u32)ent;
            act = take_item<ASTAR>(p, s, gi, K_LIGHT, L, u, ib, du, ub, inst, eb, ee, false, 0u, 0u,
                                   (u32)(ent >> 32));
            if (MAP == 2 && act && ee - eb > p.hub_min_warp) {
                // long rows: hub records beyond the CTA tier (other CTAs help), row tasks
                // of this CTA below it; the warp relaxes the row itself only when both are full
                if (p.hubs && ee - eb > p.hub_min) rec = hub_publish_at(p, s, gi, eb, ee);
                if (rec != ~0u || task_post(cs, gi, u, du, ib, inst, ub, eb, ee - eb)) act = false;
            }
        }
        if constexpr (MAP == 2) {
            // the arcs of the warp's items dealt over its lanes: the arcs of one item sit
            // in neighbouring lanes, so their loads and state updates share sectors
            relax_items_warp<ASTAR, AM>(p, s, act, u, du, ib, ub, inst, eb, ee, L, &cs);
            // hub rows this warp published: it works them itself (other CTAs' agents help)
            unsigned pubs = __ballot_sync(FULL, rec != ~0u);
            while (pubs) {
                const int l = __ffs(pubs) - 1;
                pubs &= pubs - 1u;
                u64 wub = ~0ull;
                if constexpr (ASTAR) wub = __shfl_sync(FULL, ub, l);
                warp_own_hub<ASTAR, AM>(p, s, __shfl_sync(FULL, rec, l), __shfl_sync(FULL, u, l),
                                        __shfl_sync(FULL, du, l), __shfl_sync(FULL, ib, l), wub,
                                        __shfl_sync(FULL, inst, l), L, &cs);
            }
        } else {  // thread / warp per item: warp-local, no block barrier
            relax_items<ASTAR, AM, MAP>(p, s, act, u, du, ib, ub, inst, eb, ee, L, cs, &cs, K_LIGHT);
        }
        const bool spilled = __any_sync(FULL, L.spilled != 0u);
        L.spilled = 0u;
        if (lane == 0) {
            if (spilled) __threadfence();  // ring pushes are visible before the pending work returns
            pending_done(cs, aq, n);
            if ((atomicAdd(&cs.wq_beats, 1u) & 7u) == 0u) atomicAdd(aq + AQ_BEAT, 1u);
            if (hint != ~0u) cs.wq_hint = hint;
        }
    }
    __syncthreads();  // every warp has left
}

// ---------------------------------------------------------------------------
// Naive round: every vertex whose activity bit is set relaxes all its arcs
// (Harish & Narayanan; reference naiveRelaxKernel, src/gpu_kernels.cuh:297-329).
// ---------------------------------------------------------------------------
template <bool ASTAR, int AM>
__device__ __forceinline__ void round_naive(const RunParams& p, const Snap& s, Local& L) {
    u32* mask_in = p.naive_mask[s.naive_in];
    const u32 stride = gridDim.x * blockDim.x;
    const u32 lane = threadIdx.x & 31u;
    // A* bound of this sweep (dist(target) at its start; a stale bound prunes less, never wrongly)
    u64 ub = ~0ull;
    if constexpr (ASTAR) ub = astar_bound(p, 0u, 0u);
    // Each warp owns aligned groups of 32 vertices = one mask word; the arcs of
    // the word's active vertices are dealt out over the warp's lanes, so a long
    // row is walked by 32 lanes (two arcs each per step), and a row longer than
    // 8 CTAs' worth of arcs goes to the grid tier.
    for (u32 v0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; v0 < p.n; v0 += stride) {
        const u32 word = ld_cg(mask_in + (v0 >> 5));
        if (word == 0u) continue;  // warp-uniform
        __syncwarp();
        if (lane == 0) mask_in[v0 >> 5] = 0u;
        const u32 u = v0 + lane;
        bool act = ((word >> lane) & 1u) && u < p.n;
        u32 du = INF32, eb = 0, ee = 0;
        if (act) {
            du = st_dist(ld_state(p.state + u));
            act = du != INF32;
            if constexpr (ASTAR) {
                if (act && (u64)du + h_of(p, u) >= ub) act = false;
            }
        }
        if (act) {
            eb = __ldg(p.prow + u);
            ee = __ldg(p.prow + u + 1);
            if (p.hubs && ee - eb > p.hub_min && hub_publish(p, s, u, eb, ee)) act = false;
        }
        relax_items_warp<ASTAR, AM>(p, s, act, u, du, 0u, ub, 0u, eb, ee, L, nullptr);
    }
    if (p.hubs) {
        // every CTA works the sweep's hub records before the barrier
        __shared__ u32 s_hub[8];
        if (threadIdx.x == 0) s_hub[0] = 0u;
        __syncthreads();
        while (hub_chunk<ASTAR, AM>(p, s, L, nullptr, s_hub)) {
        }
    }
}

// ---------------------------------------------------------------------------
// Compaction round (Compaction::PrefixScan): vertices flagged in the previous
// round (near_stamp == flag_epoch) are written contiguously into the near
// queue: block-wide exclusive scan of the flags, one atomicAdd per CTA chunk
// for its base. No per-push atomics.
// ---------------------------------------------------------------------------
static __device__ void round_compact(const RunParams& p, const Snap& s, Coop& cs) {
    Ctl* c = p.ctl;
    const u32 BS = blockDim.x;
    const u32 out = s.in_buf ^ 1u;
    __shared__ u32 s_base;
    for (u32 base = blockIdx.x * BS; base < p.total; base += gridDim.x * BS) {
        const u32 i = base + threadIdx.x;
        const u32 f = (i < p.total && ld_cg(p.near_stamp + i) == s.flag_epoch) ? 1u : 0u;
        u32 total = 0;
        const u32 off = block_exclusive_scan(f, cs.wsum, total);
        if (total == 0) continue;  // block-uniform
        if (threadIdx.x == 0) s_base = atomicAdd(&c->cnt[C_NEAR0 + out], total);
        __syncthreads();
        if (f) p.nearq[out][s_base + off] = i;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Learned Delta policy: 12 features -> 3 x 64 ReLU -> 16 logits; the argmax
// picks the next bucket's schedule and multiple of the automatic Delta.
// Evaluated by the CTA that runs a bucket-advance transition.
// ---------------------------------------------------------------------------
// One dense layer out[j] = act(b[j] + sum_i w[j * NI + i] * in[i]) by the
// whole CTA: G threads per neuron (a power of two dividing 32) each sum a
// strided share of the inputs, then a shuffle reduction within the group.
template <int NI, int NO, bool RELU>
__device__ __forceinline__ void policy_layer(const float* __restrict__ w, const float* __restrict__ b,
                                             const float* in, float* out) {
    const u32 t = threadIdx.x, BS = blockDim.x;
    constexpr u32 G = 4u;  // (a compile-time stride: a thread's weight loads are all in flight at once)
    const u32 part = t & (G - 1u);
    for (u32 j = t / G; j < (u32)NO; j += BS / G) {  // uniform within each warp (NO * G % 32 == 0)
        float a = 0.f;
#pragma unroll
        for (u32 i = 0; i < (u32)NI; i += G)
            if (i + part < (u32)NI) a = fmaf(__ldg(w + j * NI + i + part), in[i + part], a);
        for (u32 o = G >> 1; o > 0; o >>= 1) a += __shfl_down_sync(FULL, a, o, G);
        if (part == 0) {
            a += __ldg(b + j);
            out[j] = RELU ? (a > 0.f ? a : 0.f) : a;
        }
    }
    __syncthreads();
}

static __device__ u32 policy_pick(const PolicyNet* net, const float* feat, float* act0, float* act1) {
    const u32 t = threadIdx.x;
    __shared__ float s_in[POL_IN];
    __shared__ float s_logit[POL_OUT];
    if (t < POL_IN) s_in[t] = (feat[t] - net->in_mean[t]) * net->in_scale[t];
    __syncthreads();
    policy_layer<POL_IN, POL_H, true>(net->w1, net->b1, s_in, act0);
    policy_layer<POL_H, POL_H, true>(net->w2, net->b2, act0, act1);
    policy_layer<POL_H, POL_H, true>(net->w3, net->b3, act1, act0);
    policy_layer<POL_H, POL_OUT, false>(net->w4, net->b4, act0, s_logit);
    u32 best = 0;
    for (u32 i = 1; i < (u32)POL_OUT; ++i)
        if (s_logit[i] > s_logit[best]) best = i;
    return best;
}

// ---------------------------------------------------------------------------
// Transition, run by the CTA that arrives last at a barrier, on a copy of the
// control block in shared memory (block-uniform control flow; thread 0 owns
// the logic, the whole CTA evaluates the policy network when a bucket advance
// asks for it).
// ---------------------------------------------------------------------------
// Features of a decision point (the start of the first bucket, or a bucket
// advance). Thread 0 of the transition CTA computes the counters, then the whole
// CTA samples the frontier (frontier_sample):
//   0 log2(1 + items of the next bucket's input: the frontier)
//   1 log2(1 + items that entered the last bucket)
//   2 log2(1 + arcs scanned in the last bucket)
//   3 work ratio of the last bucket: arcs scanned / (items x average degree)
//   4 5 6 degree histogram of the sampled frontier: rows of <= 4, 5..32, > 32 slots
//   7 light fraction of the sampled rows' arcs (w <= Delta of the bucket that ended)
//   8 spread of the sampled tentative distances, (max - min) / Delta
//   9 gap between the frontier's smallest key and the window end, / avgW
//  10 log2(Delta / avgW)
//  11 log2(1 + buckets so far)
// s_flag[3..7] hand the sample over: requested, queue kind (0 near queue 0 /
// 1 far pile), far pile index, item count, Delta. With tracing on, the row is
// written to p.trace (decision k -> row k) after the sample.
static __device__ void decision_features(const RunParams& p, Ctl& sc, const Rd& r, u32 fn, u64 est, float* f,
                                         u32* s_flag, u32 far_pile) {
    const double aw = p.avg_w > 0.0 ? p.avg_w : 1.0;
    u64 edges_now = 0;
    for (int i = 0; i < 16; ++i) edges_now += sc.edge_stripe[i];
    const double arcs = (double)(edges_now - sc.bucket_edges);
    f[0] = log2f(1.f + (float)fn);
    f[1] = log2f(1.f + (float)sc.bucket_near);
    f[2] = log2f(1.f + (float)arcs);
    f[3] = fminf(64.f, (float)(arcs / fmax(1.0, (double)sc.bucket_near * fmax(1.0, p.avg_deg))));
    f[9] = (float)((double)(est > r.hi ? est - r.hi : 0ull) / aw);
    f[10] = log2f((float)((double)r.delta / aw));
    f[11] = log2f(1.f + (float)sc.buckets);
    sc.bucket_edges = edges_now;
    s_flag[3] = 1u;
    s_flag[4] = far_pile == ~0u ? 0u : 1u;
    s_flag[5] = far_pile == ~0u ? 0u : far_pile;
    s_flag[6] = fn;
    s_flag[7] = r.delta;
}

// The sampled features 4..8 of a decision point: up to 64 items of the frontier
// (evenly spaced in its queue), their row lengths, light arcs and distances.
// Called by every thread of the transition CTA.
static __device__ void frontier_sample(const RunParams& p, const u32* q, u32 cnt, u32 delta, float* f) {
    __shared__ u32 s_bin[4], s_slots, s_dmin, s_dmax;
    const u32 t = threadIdx.x;
    if (t == 0) {
        s_bin[0] = s_bin[1] = s_bin[2] = s_bin[3] = 0u;
        s_slots = 0u;
        s_dmin = INF32;
        s_dmax = 0u;
    }
    __syncthreads();
    const u32 S = min(cnt, min(64u, blockDim.x));
    if (t < S) {
        const u32 gi = ld_cg(q + (u32)(((u64)t * cnt) / S));
        u32 inst, ib, rb, u;
        decode_item(p, gi, inst, ib, rb, u);
        u32 r0, r1;
        if (p.row_stride) {
            r0 = (rb ? __ldg(p.prow + rb) : 0u) + ROW_ALIGN * u;
            r1 = r0 + ROW_ALIGN;
        } else {
            r0 = __ldg(p.prow + rb + u);
            r1 = __ldg(p.prow + rb + u + 1);
        }
        const u32 slots = r1 - r0;
        const u32 d = st_dist(ld_state(p.state + gi));  // (issued with the row's loads)
        u32 light;
        if (p.row_stride) {
            // the row's ROW_ALIGN slots in two 16-byte loads, counted directly
            const uint4* a4 = reinterpret_cast<const uint4*>(p.adj + r0);
            const uint4 q0 = __ldg(a4), q1 = __ldg(a4 + 1);
            light = (q0.y <= delta ? 1u : 0u) + (q0.w <= delta ? 1u : 0u) + (q1.y <= delta ? 1u : 0u) +
                    (q1.w <= delta ? 1u : 0u);
        } else {
            light = light_end(p.adj, r0, r1, delta) - r0;
        }
        atomicAdd(&s_bin[slots <= 4u ? 0 : (slots <= 32u ? 1 : 2)], 1u);
        atomicAdd(&s_bin[3], light);
        atomicAdd(&s_slots, slots);
        if (d != INF32) {
            atomicMin(&s_dmin, d);
            atomicMax(&s_dmax, d);
        }
    }
    __syncthreads();
    if (t == 0) {
        const float inv = S ? 1.f / (float)S : 0.f;
        f[4] = (float)s_bin[0] * inv;
        f[5] = (float)s_bin[1] * inv;
        f[6] = (float)s_bin[2] * inv;
        f[7] = s_slots ? (float)s_bin[3] / (float)s_slots : 1.f;
        f[8] = s_dmin != INF32 ? fminf(64.f, (float)(s_dmax - s_dmin) / (float)(delta ? delta : 1u)) : 0.f;
    }
    __syncthreads();
}

// Turns the bucket that starts now into an asynchronous one: every CTA scans
// its slice of the input (the far pile, or with from_near the seeds in near
// queue 0) and then drains the ring and its claimed list. Run by the
// transition thread while every other CTA waits at the barrier.
__device__ __forceinline__ void enter_async(const RunParams& p, Ctl& sc, Rd& r, u32 from_near) {
    p.aq[AQ_HEAD] = 0u;
    p.aq[AQ_TAIL] = 0u;
    p.aq[AQ_DONE] = 0u;
    p.aq[AQ_BUSY] = r.in_count ? gridDim.x : 0u;
    p.aq[AQ_IDLE] = 0u;
    if (from_near) {
        r.in_buf = 0u;
        sc.cnt[C_NEAR0] = 0u;  // the slice length travels in r.in_count
        sc.cnt[C_NEAR1] = 0u;
    }
    r.in_kind = from_near;
    r.async_bkt = 1u;
    r.phase = PH_ASYNC;
}

static __device__ void transition(const RunParams& p, Ctl& sc, u32* s_flag, float* s_feat, float* act0,
                           float* act1) {
    const u32 t = threadIdx.x;
    __shared__ u64 s_key0;
    // s_flag[0]: 0 = no bucket advance, 1 = advance with the policy, 2 = fixed Delta
    if (t == 0) {
        Rd& r = sc.rd;
        s_flag[0] = 0;
        s_flag[3] = 0;
        if (p.hubs) p.aq[AQ_HUBS] = 0u;  // hub records live for one round / bucket drain
        const u32 ph = r.phase;
        const u32 rounds = sc.rounds;
        const u32 in_buf = r.in_buf;
        const u32 out = in_buf ^ 1u;
        const u32 old_near_epoch = r.near_epoch;
        sc.rounds = rounds + 1u;
        sc.bucket_rounds += 1u;
        r.near_epoch = old_near_epoch + 1u;  // every round pushes with a fresh stamp
        bool advance = false;
        if (p.iw && ph == PH_ASYNC) {
            // independent windows: the far stamps used so far (also after a failed
            // run, so later runs never reuse them) and the window advances
            const u32 ep = ld_relaxed(p.iw_misc + IW_MAXEP);
            if (ep > r.far_epoch) r.far_epoch = ep;
            sc.buckets = ld_relaxed(p.iw_misc + IW_ADVANCES);
        }
        if (r.status != DS_OK) {
            r.phase = PH_DONE;
        } else if (rounds > sc.round_cap) {
            r.status = DS_NOT_CONVERGED;
            r.phase = PH_DONE;
        } else if (ph == PH_INIT) {
            // Stamps continue from the previous run.
            r.near_epoch = sc.near_epoch + 1u;
            r.far_epoch = sc.far_epoch + 1u;
            r.r_epoch = sc.r_epoch + 1u;
            // Seed the k sources (reference seedKernel, src/gpu_kernels.cuh:340-352).
            bool bad = false;
            for (u32 i = 0; i < p.k; ++i) {
                const u32 ni = p.inst_off ? p.inst_off[i + 1] - p.inst_off[i] : p.n;
                bad = bad || p.srcs[i] >= ni;
            }
            for (u32 i = 0; i < p.k && !bad; ++i) {
                const u32 gi = (p.inst_off ? p.inst_off[i] : i * p.n) + p.srcs[i];
                p.state[gi] = pack_state(0u, NO_PARENT);
                if (p.mode != MODE_NAIVE) p.nearq[0][i] = gi;
            }
            sc.iterations += 1u;
            if (bad) {
                r.status = DS_BAD_SOURCE;  // sources given in device memory are checked here
                r.phase = PH_DONE;
            } else if (p.mode == MODE_NAIVE) {
                const u32 src = p.srcs[0];
                atomicOr(p.naive_mask[0] + (src >> 5), 1u << (src & 31u));
                r.naive_in = 0u;
                sc.changed = 0u;
                r.in_count = p.n;
                r.phase = PH_NAIVE;
            } else {
                u64 key0 = 0;
                if (p.astar && p.use_h)
                    key0 = heuristic_value(p.x[p.srcs[0]], p.y[p.srcs[0]], p.xt, p.yt, p.hscale);
                const u64 d = r.delta;
                sc.cnt[C_NEAR0] = p.k;
                sc.cnt[C_NEAR1] = 0u;
                r.in_buf = 0u;
                r.in_count = p.k;
                r.lo = 0ull;
                r.hi = p.mode == MODE_FRONTIER ? ~0ull : (key0 / d + 1ull) * d;
                sc.bucket_near = p.k;
                sc.bucket_rounds = 0u;
                r.phase = PH_LIGHT;
                r.async_bkt = 0u;
                if (p.iw)
                    enter_iw(p, sc, r);
                else if (p.ring && !(p.mode == MODE_DELTA && p.policy))
                    enter_async(p, sc, r, 1u);
                if (p.mode == MODE_DELTA && (p.policy || p.trace)) {
                    // The first bucket is a decision point too: features of the
                    // seed window (nothing relaxed yet) and the graph.
                    decision_features(p, sc, r, p.k, key0, s_feat, s_flag, ~0u);
                    if (p.policy) {
                        s_flag[0] = 3u;  // choose the first bucket's Delta below
                        s_key0 = key0;
                    }
                }
            }
        } else if (ph == PH_NAIVE) {
            sc.iterations += 1u;
            if (sc.changed == 0u) {
                r.phase = PH_DONE;
            } else {
                sc.changed = 0u;
                r.naive_in ^= 1u;
            }
        } else if (ph == PH_COMPACT) {
            const u32 nn = sc.cnt[C_NEAR0 + out];
            if (nn) {
                sc.cnt[C_NEAR0 + in_buf] = 0u;
                r.in_buf = out;
                r.in_count = nn;
                sc.iterations += 1u;
                r.phase = PH_LIGHT;
            } else {
                r.phase = PH_DONE;
            }
        } else if (ph == PH_ASYNC) {
            // the ring is drained: light arcs of the window are done
            sc.iterations += 1u;
            if (p.iw) {
                r.phase = PH_DONE;  // (independent windows: every instance is finished)
            } else if (r.heavy && sc.cnt[C_R]) {
                r.in_count = sc.cnt[C_R];
                r.phase = PH_HEAVY;
            } else {
                advance = true;
            }
        } else if (ph == PH_LIGHT || ph == PH_SCAN) {
            const u32 nn = sc.cnt[C_NEAR0 + out];
            if (p.prefix_scan) {
                // the round just ended flagged its improved vertices with its stamp
                r.flag_epoch = old_near_epoch;
                sc.cnt[C_NEAR0 + out] = 0u;
                r.in_count = p.total;
                r.phase = PH_COMPACT;
            } else if (nn) {
                sc.cnt[C_NEAR0 + in_buf] = 0u;
                r.in_buf = out;
                r.in_count = nn;
                sc.iterations += 1u;
                sc.bucket_near += nn;
                r.phase = PH_LIGHT;
            } else if (r.heavy && sc.cnt[C_R]) {
                r.in_count = sc.cnt[C_R];
                sc.iterations += 1u;
                r.phase = PH_HEAVY;
            } else {
                advance = true;
            }
        } else if (ph == PH_HEAVY) {
            sc.cnt[C_R] = 0u;
            r.r_epoch += 1u;  // R may be refilled in this bucket (A*)
            const u32 nn = sc.cnt[C_NEAR0 + out];
            if (r.async_bkt) {
                // asynchronous buckets: heavy arcs that land inside the window
                // (A* keys) queued their heads in the ring; drain it again
                if (__ldcg(p.aq + AQ_TAIL) != __ldcg(p.aq + AQ_HEAD)) {
                    p.aq[AQ_BUSY] = 0u;
                    p.aq[AQ_IDLE] = 0u;
                    r.in_count = 0u;
                    sc.iterations += 1u;
                    r.phase = PH_ASYNC;
                } else {
                    advance = true;
                }
            } else if (nn) {
                sc.cnt[C_NEAR0 + in_buf] = 0u;
                r.in_buf = out;
                r.in_count = nn;
                sc.iterations += 1u;
                r.phase = PH_LIGHT;
            } else {
                advance = true;
            }
        }
        if (advance) {
            sc.buckets += 1u;
            const u32 fin = r.far_out;
            const u32 fn = sc.cnt[C_FAR0 + fin];
            const u64 est = sc.far_min[fin];
            if (fn == 0u || est == ~0ull) {
                r.phase = PH_DONE;
            } else {
                s_flag[0] = p.policy ? 1u : 2u;
                if (p.policy || p.trace) decision_features(p, sc, r, fn, est, s_feat, s_flag, fin);
            }
            s_flag[2] = p.inst_far_cnt ? 1u : 0u;
        } else {
            s_flag[2] = 0u;
        }
    }
    __syncthreads();
    if (s_flag[2]) {
        // Serving: at a bucket advance the near queue is empty, so a slot with
        // no item in the far pile has nothing left to relax - its target
        // distance is final (or the target is unreachable). Counts restart for
        // the next bucket (its SCAN round recounts the items it keeps).
        const bool all_done = sc.rd.phase == PH_DONE;
        for (u32 i = t; i < p.k; i += blockDim.x) {
            if (p.inst_active[i] && (all_done || p.inst_far_cnt[i] == 0u)) {
                p.inst_active[i] = 0u;
                p.inst_done[i] = sc.rounds;
            }
            p.inst_far_cnt[i] = 0u;
        }
        __threadfence();
    }
    if (s_flag[3]) {
        // the frontier sample of the decision point, then its trace row
        frontier_sample(p, s_flag[4] ? p.farq[s_flag[5]] : p.nearq[0], s_flag[6], s_flag[7], s_feat);
        const u32 row = sc.buckets;
        if (t == 0 && p.trace && row < p.trace_cap) {
            float* tr = p.trace + (size_t)row * TRACE_W;
            for (int i = 0; i < POL_IN; ++i) tr[i] = s_feat[i];
            tr[POL_IN + 0] = (float)sc.buckets;
            tr[POL_IN + 1] = (float)sc.rd.delta;
            tr[POL_IN + 2] = (float)sc.bucket_near;
            tr[POL_IN + 3] = (float)sc.bucket_rounds;
        }
    }
    const u32 need = s_flag[0];
    if (need == 1u || need == 3u) {
        const u32 cls = policy_pick(p.net, s_feat, act0, act1);
        if (t == 0) s_flag[1] = cls;
    }
    __syncthreads();
    if (t == 0) {
        Rd& r = sc.rd;
        if (need == 3u) {
            // first bucket under the policy: the aligned window holding key0
            const float dm = (float)p.delta * kPolicyMult[s_flag[1] & 7u];
            const u32 d = dm < 1.f ? 1u : (dm > 2.0e9f ? 2000000000u : (u32)dm);
            r.delta = d;
            r.heavy = d < p.maxw ? 1u : 0u;
            r.hi = (s_key0 / d + 1ull) * d;  // aligned, as a fixed-Delta run's first window
            sc.policy_calls += 1u;
            if (p.ring && s_flag[1] < 8u) enter_async(p, sc, r, 1u);
        } else if (need != 0u) {
            // Open the next bucket: the far pile collected during this bucket is
            // scanned against the window [old hi, new hi).
            u32 d = p.delta;
            if (need == 1u) {
                const float dm = (float)p.delta * kPolicyMult[s_flag[1] & 7u];
                d = dm < 1.f ? 1u : (dm > 2.0e9f ? 2000000000u : (u32)dm);
                sc.policy_calls += 1u;
            }
            const u32 fin = r.far_out;
            const u64 est = sc.far_min[fin];
            r.delta = d;
            r.heavy = d < p.maxw ? 1u : 0u;
            r.lo = r.hi;
            // aligned windows: a policy that keeps choosing class c runs exactly
            // the buckets of fixed Delta = MULTIPLIERS[c] x the automatic Delta
            r.hi = (est / d + 1ull) * d;
            r.far_in = fin;
            r.far_out = fin ^ 1u;
            sc.cnt[C_FAR0 + (fin ^ 1u)] = 0u;
            sc.far_min[fin ^ 1u] = ~0ull;
            r.far_epoch += 1u;
            r.r_epoch += 1u;
            r.in_count = sc.cnt[C_FAR0 + fin];
            sc.iterations += 1u;
            sc.bucket_rounds = 0u;
            r.phase = PH_SCAN;
            r.async_bkt = 0u;
            sc.bucket_near = 0u;  // (rounds add their near pushes to it)
            if (p.ring && (need != 1u || s_flag[1] < 8u)) {
                enter_async(p, sc, r, 0u);
                sc.bucket_near = r.in_count;
            }
        }
        // keep the persistent stamp counters in step with the round descriptor
        sc.near_epoch = r.near_epoch;
        sc.far_epoch = r.far_epoch;
        sc.r_epoch = r.r_epoch;
        // serving steps: pause when the step's round budget is spent
        if (p.step_rounds && r.phase != PH_DONE) {
            if (sc.step_left <= 1u) {
                sc.resume_phase = r.phase;
                r.phase = PH_PAUSE;
                sc.step_left = 0u;
            } else {
                sc.step_left -= 1u;
            }
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Bounded grid barrier with tickets: arrival k of the run belongs to barrier
// (k-1)/G; the CTA holding the last ticket of a barrier loads the control
// block into shared memory with parallel vector loads, runs `transition`,
// stores it back and opens the barrier. A CTA that waits longer than
// p.timeout_ns, or sees an error status, stops waiting and the kernel winds
// down; no wait is unbounded.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void grid_barrier(const RunParams& p, Snap& s, Local& L, u64* red, Ctl& sc, u32* s_flag,
                             float* s_feat, float* act0, float* act1) {
    __syncthreads();
    Ctl* c = p.ctl;
    __shared__ u32 s_last, s_gen, s_edges;
    const bool count_edges = p.policy || p.trace;
    if (count_edges) {
        // Arcs scanned this round (for the policy's per-bucket work feature): each
        // thread's count since the last flush, summed per warp, then per CTA.
        if (threadIdx.x == 0) s_edges = 0u;
        __syncthreads();
        u32 x = L.edges - L.edges_flushed;
        L.edges_flushed = L.edges;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL, x, o);
        if ((threadIdx.x & 31u) == 0 && x) atomicAdd(&s_edges, x);
    }
    const u64 fmin = block_min_u64(L.fmin, red);  // (its barrier also completes the sums above)
    L.fmin = ~0ull;
    if (count_edges && threadIdx.x == 0 && s_edges)
        atomicAdd((unsigned long long*)&c->edge_stripe[blockIdx.x & 15u], (unsigned long long)s_edges);
    if (threadIdx.x == 0) {
        if (fmin != ~0ull) atomicMin((unsigned long long*)&c->far_min[s.far_out], (unsigned long long)fmin);
        __threadfence();
        const u32 ticket = atomicAdd(&c->bar_count, 1u);
        const u32 gen = ticket / gridDim.x;
        s_gen = gen;
        s_last = (ticket + 1u == (gen + 1u) * gridDim.x) ? 1u : 0u;
        if (s_last) __threadfence();
    }
    __syncthreads();
    constexpr u32 NCH = sizeof(Ctl) / 16;
    if (s_last) {
        for (u32 i = threadIdx.x; i < NCH; i += blockDim.x)
            reinterpret_cast<uint4*>(&sc)[i] = __ldcg(reinterpret_cast<const uint4*>(c) + i);
        __syncthreads();
        transition(p, sc, s_flag, s_feat, act0, act1);
        for (u32 i = 1 + threadIdx.x; i < NCH; i += blockDim.x) {
            __stcg(reinterpret_cast<uint4*>(c) + i, reinterpret_cast<const uint4*>(&sc)[i]);
            __threadfence();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicExch(&c->bar_gen, s_gen + 1u);
            s = sc.rd;
        }
    } else if (threadIdx.x == 0) {
        u64 t0 = global_timer_ns();
        u32 beat = p.aq ? ld_relaxed(p.aq + AQ_BEAT) : 0u;
        u32 spins = 0;
        bool ok = true;
        while (vload(&c->bar_gen) <= s_gen) {
            if ((++spins & 255u) == 0u) {
                if (vload(&c->rd.status) != DS_OK) break;
                const u64 now = global_timer_ns();
                const u32 b = p.aq ? ld_relaxed(p.aq + AQ_BEAT) : 0u;
                if (b != beat) {  // a CTA still draining its bucket made progress
                    beat = b;
                    t0 = now;
                } else if (now - t0 > p.timeout_ns) {
                    flag_timeout(c, WS_BARRIER);
                    ok = false;
                    break;
                }
                if (spins > 4096u) __nanosleep(64);
            }
        }
        __threadfence();
        const uint4* src = reinterpret_cast<const uint4*>(&c->rd);
        uint4* dst = reinterpret_cast<uint4*>(&s);
        const uint4 a0 = __ldcg(src + 0), a1 = __ldcg(src + 1), a2 = __ldcg(src + 2),
                    a3 = __ldcg(src + 3), a4 = __ldcg(src + 4);
        dst[0] = a0; dst[1] = a1; dst[2] = a2; dst[3] = a3; dst[4] = a4;
        if (!ok) s.status = DS_TIMEOUT;
    }
    if (threadIdx.x == 0 && s.status != DS_OK) s.phase = PH_DONE;
    __syncthreads();
}

// ---------------------------------------------------------------------------
// The persistent kernel.
// ---------------------------------------------------------------------------
// WD: asynchronous buckets drained by warp workers; IWK: independent bucket
// windows (hybrid mapping only, SSSP only for IWK; each its own instantiation, so
// the block-synchronous drain's code and registers stay as they are).
template <bool ASTAR, int AM, int MAP, bool WD = false, bool IWK = false>
__global__ void __maxnreg__(64) k_persistent(const __grid_constant__ RunParams p) {
    __shared__ Snap s;
    // the cooperative-mapping arrays and the claimed list live in dynamic shared
    // memory (more than the 48 KB static limit)
    extern __shared__ __align__(16) unsigned char pfg_dyn_smem[];
    Coop& cs = *reinterpret_cast<Coop*>(pfg_dyn_smem);
    __shared__ Ctl sc;
    __shared__ u64 red[32];
    __shared__ u32 s_flag[8];
    __shared__ float s_feat[POL_IN];
    __shared__ float act0[POL_H], act1[POL_H];
    Local L;
    static_assert(!IWK || (!ASTAR && MAP == 2 && !WD), "independent windows: SSSP, hybrid mapping, CTA passes");
    // Failure test: with CTA 0 absent no barrier completes; every other CTA's
    // wait runs into its time limit and the run ends with DS_TIMEOUT.
    if (p.test_absent_cta && blockIdx.x == 0) return;

    if (p.resume) {
        // Continue a paused machine (serving): the round descriptor in the
        // control block is already set for the next round.
        if (threadIdx.x == 0) {
            const uint4* src = reinterpret_cast<const uint4*>(&p.ctl->rd);
            uint4* dst = reinterpret_cast<uint4*>(&s);
            for (int i = 0; i < 5; ++i) dst[i] = __ldcg(src + i);
            cs.cl_n = 0;
            cs.cl_head = 0;
            if (s.status != DS_OK) s.phase = PH_DONE;
        }
        __syncthreads();
    } else {
        // INIT: every state word to (INF, NO_PARENT) (reference initStateKernel,
        // src/gpu_kernels.cuh:334-337).
        const u64 gtid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
        const u64 gstride = (u64)gridDim.x * blockDim.x;
        for (u64 i = gtid; i < p.total; i += gstride) p.state[i] = STATE_INIT;
        if (threadIdx.x == 0) {
            s.far_out = 0;
            cs.cl_n = 0;
            cs.cl_head = 0;
        }
        grid_barrier(p, s, L, red, sc, s_flag, s_feat, act0, act1);
    }

    while (s.phase != PH_DONE && s.phase != PH_PAUSE) {
        const u32 ph = s.phase;
        if (ph == PH_LIGHT) {
            round_items<ASTAR, AM, MAP>(p, s, p.nearq[s.in_buf], s.in_count, K_LIGHT, L, cs);
        } else if (ph == PH_SCAN) {
            round_items<ASTAR, AM, MAP>(p, s, p.farq[s.far_in], s.in_count, K_SCAN, L, cs);
        } else if (ph == PH_HEAVY) {
            round_items<ASTAR, AM, MAP>(p, s, p.rq, s.in_count, K_HEAVY, L, cs);
        } else if (ph == PH_NAIVE) {
            round_naive<ASTAR, AM>(p, s, L);
        } else if (ph == PH_COMPACT) {
            round_compact(p, s, cs);
        } else if (ph == PH_ASYNC && IWK) {
            if constexpr (IWK) inst_drain<AM>(p, s, L, cs);
        } else if (ph == PH_ASYNC) {
            if constexpr (WD) wq_reset(cs);
            if (s.in_count) {
                // bucket start: this CTA's slice of the far pile (in-window items
                // are relaxed at once, the rest stay far) or of the seeds
                if (s.in_kind)
                    round_items<ASTAR, AM, MAP>(p, s, p.nearq[s.in_buf], s.in_count, K_LIGHT, L, cs);
                else
                    round_items<ASTAR, AM, MAP>(p, s, p.farq[s.far_in], s.in_count, K_SCAN, L, cs);
            }
            // (the transition gave every CTA a busy unit when there is a slice to scan)
            if constexpr (WD)
                warp_drain<ASTAR, AM, MAP>(p, s, L, cs, s.in_count != 0u);
            else
                async_drain<ASTAR, AM, MAP>(p, s, L, cs, s.in_count != 0u);
        }
        grid_barrier(p, s, L, red, sc, s_flag, s_feat, act0, act1);
    }

    // Counters summed per warp, then per CTA: one atomicAdd per CTA and counter.
    __shared__ unsigned long long s_st[4];
    if (threadIdx.x < 4u) s_st[threadIdx.x] = 0ull;
    __syncthreads();
    unsigned long long a = L.edges, b = L.atomics, cc = L.updates, d = L.pushes;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(FULL, a, o);
        b += __shfl_down_sync(FULL, b, o);
        cc += __shfl_down_sync(FULL, cc, o);
        d += __shfl_down_sync(FULL, d, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        if (a) atomicAdd(&s_st[0], a);
        if (b) atomicAdd(&s_st[1], b);
        if (cc) atomicAdd(&s_st[2], cc);
        if (d) atomicAdd(&s_st[3], d);
    }
    __syncthreads();
    if (threadIdx.x < 4u && s_st[threadIdx.x]) atomicAdd(&p.ctl->stats[threadIdx.x], s_st[threadIdx.x]);
}

}  // namespace pfg

