// gpu_solver.cpp - the C++ GpuSolver on top of the C ABI (include/pfg.h).
//
// Plain host C++ (no CUDA headers): a drop-in for the reference's
// src/gpu_sssp.cu + src/gpu_device.cu. Semantics kept from the reference
// (src/gpu_sssp.cu:461-569): sssp() unpacks dist/parent when copyBack is
// set; astar() returns the target distance and the path rebuilt from the
// parent pointers; multiSource() returns one dist vector per source and drops
// parents; errors throw std::runtime_error with the engine's message.
#include "gpu_sssp.h"
#include "pfg.h"

#include <algorithm>
#include <stdexcept>
#include <string>

namespace {

void check(pfg_status st) {
    if (st != PFG_OK) throw std::runtime_error(pfg_last_error());
}

pfg_options to_c(const GpuOptions& o) {
    pfg_options c;
    c.algo = static_cast<int32_t>(o.algo);
    c.mapping = static_cast<int32_t>(o.mapping);
    c.atomic = static_cast<int32_t>(o.atomic);
    c.delta = o.delta;
    c.block_size = o.blockSize;
    c.sync_every = o.syncEvery;
    c.compaction = static_cast<int32_t>(o.compaction);
    c.policy = PFG_POLICY_FIXED;
    c.eager = -1;
    c.blocks_per_sm = 0;
    c.schedule = PFG_SCHEDULE_AUTO;
    return c;
}

void to_cpp(const pfg_stats& s, GpuStats& o) {
    o.edgesScanned = s.edges_scanned;
    o.atomicsIssued = s.atomics_issued;
    o.updates = s.updates;
    o.pushes = s.pushes;
    o.iterations = s.iterations;
    o.hostSyncs = s.host_syncs;
    o.launches = s.launches;
    o.buckets = s.buckets;
    o.delta = s.delta;
}

// Parent chain dst -> src, reversed; empty when broken (same contract as the
// reference's reconstructPath, src/cpu_sssp.cpp:124-135).
std::vector<u32> walk_parents(const std::vector<u32>& parent, u32 src, u32 dst) {
    std::vector<u32> path;
    if (dst >= parent.size()) return path;
    u32 v = dst;
    for (size_t steps = 0; steps <= parent.size(); ++steps) {
        path.push_back(v);
        if (v == src) {
            std::reverse(path.begin(), path.end());
            return path;
        }
        v = parent[v];
        if (v == NO_PARENT || v >= parent.size()) break;
    }
    return {};
}

}  // namespace

const char* toString(GpuAlgo a) {
    switch (a) {
        case GpuAlgo::NaiveRelax: return "Naive-Relax";
        case GpuAlgo::Frontier: return "Frontier";
        case GpuAlgo::DeltaStep: return "Delta-Step";
    }
    return "?";
}
const char* toString(Compaction c) { return c == Compaction::PrefixScan ? "prefix-sum" : "warp-atomic"; }
const char* toString(Mapping m) {
    switch (m) {
        case Mapping::Thread: return "thread";
        case Mapping::Warp: return "warp";
        case Mapping::Hybrid: return "hybrid";
    }
    return "?";
}
const char* toString(AtomicMode a) {
    switch (a) {
        case AtomicMode::MinRBA: return "atomicMin+RBA";
        case AtomicMode::CasRBA: return "atomicCAS+RBA";
        case AtomicMode::MinNoCheck: return "atomicMin(no-check)";
    }
    return "?";
}

GpuDeviceInfo gpuQueryDevice(int dev) {
    GpuDeviceInfo info;
    pfg_device_info d;
    if (pfg_query_device(dev, &d) != PFG_OK || !d.ok) return info;
    info.ok = true;
    info.name = d.name;
    info.ccMajor = d.cc_major;
    info.ccMinor = d.cc_minor;
    info.smCount = d.sm_count;
    info.clockMHz = d.clock_mhz;
    info.memClockMHz = d.mem_clock_mhz;
    info.busWidth = d.bus_width;
    info.driverVersion = d.driver_version;
    info.runtimeVersion = d.runtime_version;
    info.maxThreadsPerSM = d.max_threads_per_sm;
    info.warpSize = d.warp_size;
    info.globalMem = (size_t)d.global_mem;
    info.sharedPerBlock = (size_t)d.shared_per_block;
    info.l2Bytes = (size_t)d.l2_bytes;
    info.peakBandwidthGBs = d.peak_bandwidth_gbs;
    return info;
}

void gpuWarmup() { check(pfg_warmup()); }

TransferStudy gpuTransferStudy(const CSRGraph& g, int reps) {
    pfg_transfer_study t;
    check(pfg_transfer_study_run(g.row_offsets.data(), g.col_indices.data(), g.weights.data(), g.n,
                                 g.m, reps, &t));
    TransferStudy r;
    r.bytes = t.bytes;
    r.pageableMs = t.pageable_ms;
    r.pinnedMs = t.pinned_ms;
    r.pinnedStreamsMs = t.pinned_streams_ms;
    return r;
}

struct GpuSolver::Impl {
    const CSRGraph& g;  // the caller's graph must outlive the solver (as in the reference)
    pfg_solver* h = nullptr;
    u32 K = 1;
    std::vector<u64> state;

    Impl(const CSRGraph& graph, u32 maxBatch) : g(graph), K(std::max<u32>(1, maxBatch)) {
        const bool xy = graph.hasCoords();
        check(pfg_create(graph.row_offsets.data(), graph.col_indices.data(), graph.weights.data(),
                         xy ? graph.x.data() : nullptr, xy ? graph.y.data() : nullptr, graph.n,
                         graph.m, graph.hScale, graph.avgW, graph.avgDeg, K, &h));
    }
    ~Impl() { pfg_destroy(h); }

    GpuRunResult run(const u32* srcs, u32 k, bool astar, u32 dst, const GpuOptions& o, bool copyBack) {
        GpuRunResult r;
        pfg_options c = to_c(o);
        pfg_stats st;
        float ms = 0.f;
        const bool need_state = copyBack || astar;
        if (need_state) state.resize((size_t)k * g.n);
        check(pfg_run(h, srcs, k, astar ? 1 : 0, dst, &c, &st, need_state ? state.data() : nullptr, &ms));
        r.ms = ms;
        to_cpp(st, r.stats);
        if (!need_state) return r;
        if (astar) {
            std::vector<u32> parent(g.n);
            for (u32 v = 0; v < g.n; ++v) parent[v] = (u32)(state[v] & 0xFFFFFFFFull);
            r.targetDist = (u32)(state[dst] >> 32);
            if (r.targetDist != INF_DIST) r.path = walk_parents(parent, srcs[0], dst);
        } else if (k == 1) {
            r.dist.resize(g.n);
            r.parent.resize(g.n);
            for (u32 v = 0; v < g.n; ++v) {
                r.dist[v] = (u32)(state[v] >> 32);
                r.parent[v] = (u32)(state[v] & 0xFFFFFFFFull);
            }
        }
        return r;
    }
};

GpuSolver::GpuSolver(const CSRGraph& g, u32 maxBatch) : p_(new Impl(g, maxBatch)) {}
GpuSolver::~GpuSolver() { delete p_; }
double GpuSolver::uploadMs() const { return pfg_upload_ms(p_->h); }
size_t GpuSolver::deviceBytes() const { return (size_t)pfg_device_bytes(p_->h); }
u32 GpuSolver::autoDelta() const { return pfg_auto_delta(p_->h); }

GpuRunResult GpuSolver::sssp(u32 src, const GpuOptions& opt, bool copyBack) {
    return p_->run(&src, 1, false, 0, opt, copyBack);
}

GpuRunResult GpuSolver::astar(u32 src, u32 dst, const GpuOptions& opt) {
    return p_->run(&src, 1, true, dst, opt, false);
}

GpuRunResult GpuSolver::multiSource(const std::vector<u32>& srcs, const GpuOptions& opt,
                                    std::vector<std::vector<u32>>* distOut) {
    const u32 k = (u32)srcs.size();
    // k == 1 fills r.dist / r.parent as well, as the reference does; for k > 1
    // only the distances come back, split from the packed words on the device.
    GpuRunResult r = p_->run(srcs.data(), k, false, 0, opt, distOut != nullptr && k == 1);
    if (distOut) {
        const u32 n = p_->g.n;
        distOut->assign(k, std::vector<u32>(n));
        if (k == 1) {
            (*distOut)[0] = r.dist;
        } else {
            for (u32 i = 0; i < k; ++i) check(pfg_copy_dist(p_->h, (uint64_t)i * n, n, (*distOut)[i].data()));
        }
    }
    return r;
}
