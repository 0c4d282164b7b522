// gpu_sssp.h - C++ host interface of the B200 SSSP / A* engine.
//
// Source-compatible with the reference's GpuSolver interface
// (include/gpu_sssp.h:10-120 of nmd-coder/pathfinding_gpu): the same enums,
// option / statistics / result structs, free functions and class, so an
// application written against the reference (its src/main.cpp) compiles and
// links unchanged against this implementation (gpu_solver.cpp, which calls
// the C ABI of include/pfg.h). No CUDA type appears here.
//
// `CSRGraph` comes from the application's "graph.h" (the reference's
// include/graph.h, or pathfinding_gpu_b200/csrc/compat/graph.h for standalone
// builds): n, m, row_offsets, col_indices, weights (rows sorted by weight),
// x, y, hScale, avgW, avgDeg.
#pragma once
#include "graph.h"

#include <string>
#include <vector>

enum class GpuAlgo {
    NaiveRelax,  // Bellman-Ford sweep over all vertices with activity flags
    Frontier,    // frontier queue, no buckets
    DeltaStep    // Delta-stepping buckets with light / heavy arcs
};

enum class Mapping {
    Thread,  // one thread per frontier vertex
    Warp,    // one warp per frontier vertex
    Hybrid   // short rows per thread, long rows spread over the CTA
};

enum class AtomicMode {
    MinRBA,     // read the state first, atomicMin only on improvement (default)
    CasRBA,     // read first, then a compare-and-swap loop
    MinNoCheck  // blind atomicMin
};

enum class Compaction {
    WarpAtomic,  // dedup stamp + warp-aggregated queue append (default)
    PrefixScan   // flags + block scans, no per-vertex atomics (Frontier only)
};

const char* toString(Compaction c);
const char* toString(GpuAlgo a);
const char* toString(Mapping m);
const char* toString(AtomicMode a);

struct GpuOptions {
    GpuAlgo algo = GpuAlgo::DeltaStep;
    Mapping mapping = Mapping::Hybrid;
    AtomicMode atomic = AtomicMode::MinRBA;
    u32 delta = 0;      // 0: automatic, 32 * avgW / avgDeg
    int blockSize = 256;
    u32 syncEvery = 8;  // kept for compatibility; convergence is detected on the device
    Compaction compaction = Compaction::WarpAtomic;
};

struct GpuStats {
    u64 edgesScanned = 0;
    u64 atomicsIssued = 0;
    u64 updates = 0;
    u64 pushes = 0;
    u32 iterations = 0;
    u32 hostSyncs = 0;
    u32 launches = 0;
    u32 buckets = 0;
    u32 delta = 0;
};

struct GpuRunResult {
    double ms = 0.0;            // device time of init + relaxation (CUDA events)
    GpuStats stats;
    std::vector<u32> dist;      // SSSP: all vertices; A*: empty
    std::vector<u32> parent;
    u32 targetDist = INF_DIST;  // A*
    std::vector<u32> path;      // A*: src ... dst
};

struct GpuDeviceInfo {
    bool ok = false;
    std::string name;
    int ccMajor = 0, ccMinor = 0, smCount = 0, clockMHz = 0, memClockMHz = 0, busWidth = 0;
    int driverVersion = 0, runtimeVersion = 0, maxThreadsPerSM = 0, warpSize = 32;
    size_t globalMem = 0, sharedPerBlock = 0, l2Bytes = 0;
    double peakBandwidthGBs = 0.0;
};
GpuDeviceInfo gpuQueryDevice(int dev = 0);
void gpuWarmup();

struct TransferStudy {
    double bytes = 0;
    double pageableMs = 0, pinnedMs = 0, pinnedStreamsMs = 0;
};
TransferStudy gpuTransferStudy(const CSRGraph& g, int reps);

// Holds the graph and every working buffer on the device (allocated once).
// Errors throw std::runtime_error, as in the reference.
class GpuSolver {
public:
    GpuSolver(const CSRGraph& g, u32 maxBatch = 1);
    ~GpuSolver();
    GpuSolver(const GpuSolver&) = delete;
    GpuSolver& operator=(const GpuSolver&) = delete;

    double uploadMs() const;
    size_t deviceBytes() const;
    u32 autoDelta() const;

    GpuRunResult sssp(u32 src, const GpuOptions& opt, bool copyBack = true);
    GpuRunResult astar(u32 src, u32 dst, const GpuOptions& opt);
    GpuRunResult multiSource(const std::vector<u32>& srcs, const GpuOptions& opt,
                             std::vector<std::vector<u32>>* distOut);

private:
    struct Impl;
    Impl* p_;
};
