// ref_shim.cpp - TEST INFRASTRUCTURE. extern "C" entry points over the
// reference's own CPU code (graph.cpp, cpu_sssp.cpp, verify.cpp), compiled
// together with those sources by oracle/Makefile into oracle/_ref/libpfref.so.
// Used to pin the C oracle (pfg_oracle.c) and as the timed CPU baseline of
// bench.py; never part of the product.
#include "cpu_sssp.h"
#include "graph.h"
#include "heuristic.h"
#include "verify.h"

#include <algorithm>
#include <cstring>
#include <vector>

struct RefGraph {
    CSRGraph g;
};

static RefGraph* wrap(CSRGraph&& g) {
    RefGraph* r = new RefGraph();
    r->g = std::move(g);
    return r;
}

extern "C" {

void* ref_gen_grid_road(u32 rows, u32 cols, u64 seed) { return wrap(buildCSR(genGridRoad(rows, cols, seed))); }

void* ref_gen_rmat(u32 scale, u32 ef, u32 maxw, u64 seed) { return wrap(buildCSR(genRMAT(scale, ef, maxw, seed))); }

void* ref_build_csr(u32 n, u64 m, const u32* s, const u32* d, const u32* w, const double* x, const double* y) {
    EdgeList el;
    el.n = n;
    el.src.assign(s, s + m);
    el.dst.assign(d, d + m);
    el.w.assign(w, w + m);
    if (x && y) {
        el.x.assign(x, x + n);
        el.y.assign(y, y + n);
    }
    return wrap(buildCSR(std::move(el)));
}

// Wraps an existing weight-sorted CSR without rebuilding it.
void* ref_wrap_csr(u32 n, u32 m, const u32* row, const u32* col, const u32* w, const double* x,
                   const double* y, double hscale) {
    CSRGraph g;
    g.n = n;
    g.m = m;
    g.row_offsets.assign(row, row + n + 1);
    g.col_indices.assign(col, col + m);
    g.weights.assign(w, w + m);
    if (x && y) {
        g.x.assign(x, x + n);
        g.y.assign(y, y + n);
    }
    g.hScale = hscale;
    return wrap(std::move(g));
}

void ref_free(void* h) { delete (RefGraph*)h; }
u32 ref_n(void* h) { return ((RefGraph*)h)->g.n; }
u32 ref_m(void* h) { return ((RefGraph*)h)->g.m; }
const u32* ref_row(void* h) { return ((RefGraph*)h)->g.row_offsets.data(); }
const u32* ref_col(void* h) { return ((RefGraph*)h)->g.col_indices.data(); }
const u32* ref_w(void* h) { return ((RefGraph*)h)->g.weights.data(); }
const double* ref_x(void* h) { return ((RefGraph*)h)->g.x.empty() ? nullptr : ((RefGraph*)h)->g.x.data(); }
const double* ref_y(void* h) { return ((RefGraph*)h)->g.y.empty() ? nullptr : ((RefGraph*)h)->g.y.data(); }

// out: [m, minW, maxW, maxDeg, avgW, avgDeg, hScale]
void ref_stats(void* h, double* out) {
    const CSRGraph& g = ((RefGraph*)h)->g;
    out[0] = g.m; out[1] = g.minW; out[2] = g.maxW; out[3] = g.maxDeg;
    out[4] = g.avgW; out[5] = g.avgDeg; out[6] = g.hScale;
}

double ref_dijkstra(void* h, u32 src, u32* dist, u32* parent, u64* edges) {
    SSSPResult r = cpuDijkstra(((RefGraph*)h)->g, src);
    if (dist) std::copy(r.dist.begin(), r.dist.end(), dist);
    if (parent) std::copy(r.parent.begin(), r.parent.end(), parent);
    if (edges) *edges = r.edgesScanned;
    return r.ms;
}

u32 ref_astar(void* h, u32 src, u32 dst, int use_h, u32* path, u32* path_len, double* ms, u64* edges) {
    P2PResult r = cpuAStar(((RefGraph*)h)->g, src, dst, use_h != 0);
    if (path) std::copy(r.path.begin(), r.path.end(), path);
    if (path_len) *path_len = (u32)r.path.size();
    if (ms) *ms = r.ms;
    if (edges) *edges = r.edgesScanned;
    return r.dist;
}

double ref_multi_source(void* h, const u32* srcs, u32 k, int threads, u32* dist_out, u64* edges) {
    std::vector<u32> s(srcs, srcs + k);
    MultiSourceCpuResult r = cpuMultiSource(((RefGraph*)h)->g, s, threads, dist_out != nullptr);
    if (dist_out) {
        const u32 n = ((RefGraph*)h)->g.n;
        for (u32 i = 0; i < k; ++i) std::copy(r.dist[i].begin(), r.dist[i].end(), dist_out + (size_t)i * n);
    }
    if (edges) *edges = r.edgesScanned;
    return r.ms;
}

int ref_max_threads(void) { return cpuMaxThreads(); }

u64 ref_verify_sssp(void* h, u32 src, const u32* ref_dist, const u32* dist, const u32* parent,
                    u32 samples, u64 seed, u64* report) {
    const CSRGraph& g = ((RefGraph*)h)->g;
    std::vector<u32> rd(ref_dist, ref_dist + g.n), d(dist, dist + g.n), p(parent, parent + g.n);
    VerifyReport v = verifySSSP(g, src, rd, d, p, samples, seed);
    report[0] = v.distChecked; report[1] = v.distMismatch; report[2] = v.treeChecked;
    report[3] = v.treeErrors; report[4] = v.pathsChecked; report[5] = v.pathErrors;
    return v.totalErrors();
}

int ref_validate_path(void* h, const u32* path, u32 len, u32 src, u32 dst, u32 expected) {
    std::vector<u32> p(path, path + len);
    return validatePath(((RefGraph*)h)->g, p, src, dst, expected, nullptr) ? 1 : 0;
}

void ref_pick_sources(void* h, u32 count, u64 seed, u32* out) {
    std::vector<u32> s = pickSources(((RefGraph*)h)->g, count, seed);
    std::copy(s.begin(), s.end(), out);
}

// The reference's loaders (graph.cpp: loadDIMACS, loadSNAP, loadBinary,
// saveBinary); a loaded edge list goes through buildCSR as in its main.cpp.
// NULL (or 0) when the reference's loader reports failure.
void* ref_load_dimacs(const char* gr, const char* co) {
    EdgeList el;
    if (!loadDIMACS(gr, co ? co : "", el)) return nullptr;
    return wrap(buildCSR(std::move(el)));
}

void* ref_load_snap(const char* path, int symmetrize, u32 maxw, u64 seed) {
    EdgeList el;
    if (!loadSNAP(path, symmetrize != 0, maxw, seed, el)) return nullptr;
    return wrap(buildCSR(std::move(el)));
}

void* ref_load_binary(const char* path) {
    CSRGraph g;
    if (!loadBinary(path, g)) return nullptr;
    return wrap(std::move(g));
}

int ref_save_binary(void* h, const char* path) { return saveBinary(((RefGraph*)h)->g, path) ? 1 : 0; }

u32 ref_heuristic(double xv, double yv, double xt, double yt, double scale) {
    return heuristicValue(xv, yv, xt, yt, scale);
}

}  // extern "C"
