/*
 * pfg_oracle.c - CPU ORACLE (test infrastructure only).
 *
 * A plain C restatement of the reference's CPU algorithms for the SSSP / A*
 * path. It is the checker of the CUDA engine: only the tests, the smoke test
 * and the CPU legs of bench.py load it; the product never links it.
 *
 * Pinned against the reference itself: tests/golden/make_golden.py runs the
 * reference's own cpuDijkstra / cpuAStar / buildCSR / genGridRoad / genRMAT
 * (compiled from its sources by oracle/Makefile into oracle/_ref) and stores
 * their outputs as fixtures; tests/test_oracle.py checks this file against
 * those fixtures and against the graph statistics the reference printed in
 * its published logs (results/colab_T4/logs/verify_grid_1e6.txt:7-10,
 * results/colab_T4/logs/bench_rmat.txt:75-77).
 *
 * Functions and the reference code they restate:
 *   orc_rng_*            Rng (SplitMix64)               include/common.h:44-56
 *   orc_hash64           hash64                         include/common.h:58-62
 *   orc_heuristic        heuristicValue                 include/heuristic.h:19-25
 *   orc_build_csr        buildCSR                       src/graph.cpp:23-104
 *   orc_gen_grid_road    genGridRoad                    src/graph.cpp:113-152
 *   orc_gen_rmat_ref     genRMAT                        src/graph.cpp:158-199
 *   orc_dijkstra         cpuDijkstra                    src/cpu_sssp.cpp:28-57
 *   orc_min_parent       smallest tight predecessor: the parent the packed
 *                        (dist<<32|parent) atomicMin of the GPU converges to
 *                        (src/gpu_kernels.cuh:11-13, 96-121)
 *   orc_astar            cpuAStar                       src/cpu_sssp.cpp:64-101
 *   orc_multi_source     cpuMultiSource (OpenMP)        src/cpu_sssp.cpp:103-122
 *   orc_reconstruct_path reconstructPath                src/cpu_sssp.cpp:124-135
 *   orc_validate_path    validatePath                   src/verify.cpp:25-52
 *   orc_verify_sssp      verifySSSP checks (1)-(3)      src/verify.cpp:54-99
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint32_t u32;
typedef uint64_t u64;
#define INF32 0xFFFFFFFFu

/* ---------------- SplitMix64 (reference Rng seeding) ---------------- */
typedef struct { u64 s; } orc_rng;
static void rng_init(orc_rng* r, u64 seed) { r->s = seed * 0x9E3779B97F4A7C15ull + 0x1234567ull; }
static u64 rng_next(orc_rng* r) {
    u64 z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_uniform(orc_rng* r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static double rng_uniform_ab(orc_rng* r, double a, double b) { return a + (b - a) * rng_uniform(r); }
static u32 rng_below(orc_rng* r, u32 n) { return (u32)(rng_next(r) % n); }

u64 orc_rng_stream(u64 seed, u64 count, u64* out) {
    orc_rng r;
    rng_init(&r, seed);
    for (u64 i = 0; i < count; ++i) out[i] = rng_next(&r);
    return count;
}
u64 orc_hash64(u64 x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33; return x;
}

/* ---------------- heuristic ---------------- */
u32 orc_heuristic(double xv, double yv, double xt, double yt, double scale) {
    double dx = xv - xt, dy = yv - yt;
    double e = sqrt(dx * dx + dy * dy) * scale * (1.0 - 1e-9);
    if (!(e > 0.0)) return 0u;
    if (e >= 4.0e9) return 4000000000u;
    return (u32)e;
}

/* ---------------- CSR builder ---------------- */
static int cmp_u64(const void* a, const void* b) {
    u64 x = *(const u64*)a, y = *(const u64*)b;
    return x < y ? -1 : x > y;
}

/* stats_out: [m, minW, maxW, maxDeg, avgW, avgDeg, hScale]. Returns 0 or -1. */
int orc_build_csr(u32 n, u64 m_in, const u32* src, const u32* dst, const u32* w, const double* x,
                  const double* y, u32* row, u32* col, u32* wt, double* stats_out) {
    u32* deg = (u32*)calloc((size_t)n + 1, sizeof(u32));
    u64 keep = 0;
    for (u64 i = 0; i < m_in; ++i)
        if (src[i] != dst[i]) { deg[src[i]]++; keep++; }
    if (keep >= 0xFFFFFFFFull) { free(deg); return -1; }
    u32 m = (u32)keep;
    row[0] = 0;
    for (u32 u = 0; u < n; ++u) row[u + 1] = row[u] + deg[u];
    u32* cur = deg; /* reuse as cursor */
    for (u32 u = 0; u < n; ++u) cur[u] = row[u];
    for (u64 i = 0; i < m_in; ++i) {
        u32 s = src[i], d = dst[i];
        if (s == d) continue;
        u32 pos = cur[s]++;
        col[pos] = d;
        wt[pos] = w[i] < 1u ? 1u : w[i];
    }
    free(deg);
    u64* tmp = NULL;
    size_t cap = 0;
    for (u32 u = 0; u < n; ++u) {
        u32 b = row[u], e = row[u + 1];
        if (e - b < 2) continue;
        if (cap < e - b) { cap = e - b; tmp = (u64*)realloc(tmp, cap * sizeof(u64)); }
        for (u32 k = b; k < e; ++k) tmp[k - b] = ((u64)wt[k] << 32) | col[k];
        qsort(tmp, e - b, sizeof(u64), cmp_u64);
        for (u32 k = b; k < e; ++k) { wt[k] = (u32)(tmp[k - b] >> 32); col[k] = (u32)tmp[k - b]; }
    }
    free(tmp);
    u32 minw = m ? 0xFFFFFFFFu : 0u, maxw = 0, maxdeg = 0;
    double sum = 0.0;
    for (u32 k = 0; k < m; ++k) {
        if (wt[k] < minw) minw = wt[k];
        if (wt[k] > maxw) maxw = wt[k];
        sum += wt[k];
    }
    for (u32 u = 0; u < n; ++u) if (row[u + 1] - row[u] > maxdeg) maxdeg = row[u + 1] - row[u];
    double hs = 0.0;
    if (x && y) {
        double scale = INFINITY;
        for (u32 u = 0; u < n; ++u)
            for (u32 k = row[u]; k < row[u + 1]; ++k) {
                u32 v = col[k];
                double dx = x[u] - x[v], dy = y[u] - y[v];
                double e = sqrt(dx * dx + dy * dy);
                if (e > 1e-12 && wt[k] / e < scale) scale = wt[k] / e;
            }
        hs = isfinite(scale) ? scale : 0.0;
    }
    stats_out[0] = m; stats_out[1] = minw; stats_out[2] = maxw; stats_out[3] = maxdeg;
    stats_out[4] = m ? sum / m : 0.0; stats_out[5] = n ? (double)m / n : 0.0; stats_out[6] = hs;
    return 0;
}

/* ---------------- reference generators (restated, for pins) ---------------- */
/* Arc capacity needed: 8 * rows * cols. Returns the arc count. */
u64 orc_gen_grid_road(u32 rows, u32 cols, u64 seed, u32* s, u32* d, u32* w, double* x, double* y) {
    orc_rng r;
    rng_init(&r, seed);
    for (u32 a = 0; a < rows; ++a)
        for (u32 c = 0; c < cols; ++c) {
            u32 id = a * cols + c;
            x[id] = c * 100.0 + rng_uniform_ab(&r, -25.0, 25.0);
            y[id] = a * 100.0 + rng_uniform_ab(&r, -25.0, 25.0);
        }
    u64 m = 0;
#define ROAD(A, B, ART)                                                             \
    do {                                                                            \
        double dx_ = x[A] - x[B], dy_ = y[A] - y[B];                                \
        double e_ = sqrt(dx_ * dx_ + dy_ * dy_);                                    \
        double f_ = (ART) ? rng_uniform_ab(&r, 1.0, 1.15) : rng_uniform_ab(&r, 1.15, 1.9); \
        long long q_ = llround(e_ * f_);                                            \
        u32 w_ = (u32)(q_ < 1 ? 1 : q_);                                            \
        s[m] = (A); d[m] = (B); w[m] = w_; ++m;                                     \
        s[m] = (B); d[m] = (A); w[m] = w_; ++m;                                     \
    } while (0)
    for (u32 a = 0; a < rows; ++a)
        for (u32 c = 0; c < cols; ++c) {
            u32 id = a * cols + c;
            if (c + 1 < cols) {
                int art = (a % 16 == 0);
                if (art || rng_uniform(&r) < 0.95) ROAD(id, id + 1, art);
            }
            if (a + 1 < rows) {
                int art = (c % 16 == 0);
                if (art || rng_uniform(&r) < 0.95) ROAD(id, id + cols, art);
            }
            if (a + 1 < rows && c + 1 < cols && rng_uniform(&r) < 0.05) ROAD(id, id + cols + 1, 0);
            if (a + 1 < rows && c > 0 && rng_uniform(&r) < 0.05) ROAD(id, id + cols - 1, 0);
        }
#undef ROAD
    return m;
}

/* Undirected, label-permuted R-MAT with hash weights. Arc capacity needed:
 * 2 * edge_factor * 2^scale. Returns the arc count. */
u64 orc_gen_rmat_ref(u32 scale, u32 ef, u32 maxw, u64 seed, u32* s, u32* d, u32* w) {
    u32 n = 1u << scale;
    u64 target = (u64)n * ef;
    const double A = 0.57, B = 0.19, C = 0.19;
    orc_rng r;
    rng_init(&r, seed);
    u32* perm = (u32*)malloc((size_t)n * sizeof(u32));
    for (u32 i = 0; i < n; ++i) perm[i] = i;
    for (u32 i = n - 1; i > 0; --i) {
        u32 j = rng_below(&r, i + 1);
        u32 t = perm[i]; perm[i] = perm[j]; perm[j] = t;
    }
    u64* keys = (u64*)malloc((size_t)target * sizeof(u64));
    u64 nk = 0;
    for (u64 e = 0; e < target; ++e) {
        u32 u = 0, v = 0;
        for (u32 b = 0; b < scale; ++b) {
            double x = rng_uniform(&r);
            u32 bu = 0, bv = 0;
            if (x < A) {
            } else if (x < A + B) bv = 1;
            else if (x < A + B + C) bu = 1;
            else { bu = 1; bv = 1; }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        u = perm[u]; v = perm[v];
        if (u == v) continue;
        if (u > v) { u32 t = u; u = v; v = t; }
        keys[nk++] = ((u64)u << 32) | v;
    }
    free(perm);
    qsort(keys, nk, sizeof(u64), cmp_u64);
    u64 m = 0, uniq = 0;
    for (u64 i = 0; i < nk; ++i) {
        if (i && keys[i] == keys[i - 1]) continue;
        u64 k = keys[i];
        u32 u = (u32)(k >> 32), v = (u32)k;
        u32 ww = 1 + (u32)(orc_hash64(k ^ (seed * 0x9E37ull)) % maxw);
        s[m] = u; d[m] = v; w[m] = ww; ++m;
        s[m] = v; d[m] = u; w[m] = ww; ++m;
        ++uniq;
    }
    free(keys);
    (void)uniq;
    return m;
}

/* ---------------- binary heaps ---------------- */
typedef struct { u64* a; size_t n, cap; } heap64;
static void h64_push(heap64* h, u64 k) {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->a = (u64*)realloc(h->a, h->cap * sizeof(u64)); }
    size_t i = h->n++;
    while (i) { size_t p = (i - 1) / 2; if (h->a[p] <= k) break; h->a[i] = h->a[p]; i = p; }
    h->a[i] = k;
}
static u64 h64_pop(heap64* h) {
    u64 top = h->a[0], last = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1;
        if (l >= h->n) break;
        size_t c = (l + 1 < h->n && h->a[l + 1] < h->a[l]) ? l + 1 : l;
        if (h->a[c] >= last) break;
        h->a[i] = h->a[c]; i = c;
    }
    if (h->n) h->a[i] = last;
    return top;
}

typedef struct { u64 f; u32 v; } fv;
typedef struct { fv* a; size_t n, cap; } heapfv;
static int fv_less(fv x, fv y) { return x.f < y.f || (x.f == y.f && x.v < y.v); }
static void hfv_push(heapfv* h, fv k) {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->a = (fv*)realloc(h->a, h->cap * sizeof(fv)); }
    size_t i = h->n++;
    while (i) { size_t p = (i - 1) / 2; if (!fv_less(k, h->a[p])) break; h->a[i] = h->a[p]; i = p; }
    h->a[i] = k;
}
static fv hfv_pop(heapfv* h) {
    fv top = h->a[0], last = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1;
        if (l >= h->n) break;
        size_t c = (l + 1 < h->n && fv_less(h->a[l + 1], h->a[l])) ? l + 1 : l;
        if (!fv_less(h->a[c], last)) break;
        h->a[i] = h->a[c]; i = c;
    }
    if (h->n) h->a[i] = last;
    return top;
}

/* ---------------- Dijkstra ---------------- */
/* counters_out (nullable): [edges scanned, settled]. Returns elapsed ms. */
double orc_dijkstra(u32 n, const u32* row, const u32* col, const u32* wt, u32 src, u32* dist,
                    u32* parent, u64* counters_out) {
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (u32 i = 0; i < n; ++i) { dist[i] = INF32; parent[i] = INF32; }
    heap64 h = {0, 0, 0};
    u64 edges = 0, settled = 0;
    dist[src] = 0;
    h64_push(&h, (u64)src);
    while (h.n) {
        u64 top = h64_pop(&h);
        u32 d = (u32)(top >> 32), u = (u32)top;
        if (d > dist[u]) continue; /* stale entry */
        settled++;
        for (u32 k = row[u]; k < row[u + 1]; ++k) {
            u32 v = col[k];
            u64 nd = (u64)d + wt[k];
            edges++;
            if (nd < dist[v]) {
                dist[v] = (u32)nd;
                parent[v] = u;
                h64_push(&h, (nd << 32) | v);
            }
        }
    }
    free(h.a);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (counters_out) { counters_out[0] = edges; counters_out[1] = settled; }
    return (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6;
}

/* Canonical parent: the smallest u with dist[u] finite and dist[u] + w(u,v) == dist[v]. */
void orc_min_parent(u32 n, const u32* row, const u32* col, const u32* wt, const u32* dist, u32 src,
                    u32* parent) {
    for (u32 i = 0; i < n; ++i) parent[i] = INF32;
    for (u32 u = 0; u < n; ++u) {
        if (dist[u] == INF32) continue;
        for (u32 k = row[u]; k < row[u + 1]; ++k) {
            u32 v = col[k];
            if (v == src) continue;
            if ((u64)dist[u] + wt[k] == (u64)dist[v] && u < parent[v]) parent[v] = u;
        }
    }
}

/* ---------------- A* ---------------- */
u32 orc_reconstruct_path(const u32* parent, u32 n, u32 src, u32 dst, u32* path, u32 cap) {
    if (dst >= n) return 0;
    u32 v = dst, len = 0;
    for (u64 steps = 0; steps <= n; ++steps) {
        if (len >= cap) return 0;
        path[len++] = v;
        if (v == src) {
            for (u32 i = 0; i < len / 2; ++i) { u32 t = path[i]; path[i] = path[len - 1 - i]; path[len - 1 - i] = t; }
            return len;
        }
        v = parent[v];
        if (v == INF32 || v >= n) break;
    }
    return 0;
}

/* Returns the target distance; path (cap >= n) and *path_len get the path.
 * counters_out (nullable): [edges scanned, settled, elapsed ns]. */
u32 orc_astar(u32 n, const u32* row, const u32* col, const u32* wt, const double* x, const double* y,
              double hscale, u32 src, u32 dst, int use_heuristic, u32* path, u32* path_len,
              u64* counters_out) {
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    const int useH = use_heuristic && x && y && hscale > 0.0;
    const double xt = useH ? x[dst] : 0.0, yt = useH ? y[dst] : 0.0;
#define H(v) (useH ? (u64)orc_heuristic(x[v], y[v], xt, yt, hscale) : 0ull)
    u32* dist = (u32*)malloc((size_t)n * sizeof(u32));
    u32* parent = (u32*)malloc((size_t)n * sizeof(u32));
    for (u32 i = 0; i < n; ++i) { dist[i] = INF32; parent[i] = INF32; }
    heapfv h = {0, 0, 0};
    u64 edges = 0, settled = 0;
    dist[src] = 0;
    fv s0 = {H(src), src};
    hfv_push(&h, s0);
    while (h.n) {
        fv it = hfv_pop(&h);
        u32 u = it.v;
        u64 du = dist[u];
        if (it.f > du + H(u)) continue; /* stale entry */
        settled++;
        if (u == dst) break;
        for (u32 k = row[u]; k < row[u + 1]; ++k) {
            u32 v = col[k];
            u64 nd = du + wt[k];
            edges++;
            if (nd < dist[v]) {
                dist[v] = (u32)nd;
                parent[v] = u;
                fv nx = {nd + H(v), v};
                hfv_push(&h, nx);
            }
        }
    }
#undef H
    u32 td = dist[dst];
    *path_len = td != INF32 ? orc_reconstruct_path(parent, n, src, dst, path, n) : 0;
    free(h.a);
    free(dist);
    free(parent);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (counters_out) {
        counters_out[0] = edges;
        counters_out[1] = settled;
        counters_out[2] = (u64)((t1.tv_sec - t0.tv_sec) * 1000000000ll + (t1.tv_nsec - t0.tv_nsec));
    }
    return td;
}

/* ---------------- multi-source (OpenMP over sources) ---------------- */
/* dist_out (nullable): k * n distances. Returns elapsed ms. */
double orc_multi_source(u32 n, const u32* row, const u32* col, const u32* wt, const u32* srcs, u32 k,
                        int threads, u32* dist_out, u64* edges_out) {
    struct timespec t0, t1;
    u64 edges = 0;
    clock_gettime(CLOCK_MONOTONIC, &t0);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1) reduction(+ : edges)
#endif
    for (int i = 0; i < (int)k; ++i) {
        u32* d = dist_out ? dist_out + (size_t)i * n : (u32*)malloc((size_t)n * sizeof(u32));
        u32* p = (u32*)malloc((size_t)n * sizeof(u32));
        u64 c[2];
        orc_dijkstra(n, row, col, wt, srcs[i], d, p, c);
        edges += c[0];
        free(p);
        if (!dist_out) free(d);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (edges_out) *edges_out = edges;
    (void)threads;
    return (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------- verification ---------------- */
static u32 min_arc_weight(const u32* row, const u32* col, const u32* wt, u32 a, u32 b) {
    u32 best = INF32;
    for (u32 k = row[a]; k < row[a + 1]; ++k)
        if (col[k] == b && wt[k] < best) best = wt[k];
    return best;
}

/* 1 when the path src..dst exists arc by arc and costs `expected`. */
int orc_validate_path(u32 n, const u32* row, const u32* col, const u32* wt, const u32* path, u32 len,
                      u32 src, u32 dst, u32 expected) {
    (void)n;
    if (expected == INF32) return len == 0;
    if (len == 0 || path[0] != src || path[len - 1] != dst) return 0;
    u64 sum = 0;
    for (u32 i = 0; i + 1 < len; ++i) {
        u32 w = min_arc_weight(row, col, wt, path[i], path[i + 1]);
        if (w == INF32) return 0;
        sum += w;
    }
    return sum == expected;
}

/* report: [distChecked, distMismatch, treeChecked, treeErrors, pathsChecked, pathErrors].
 * Returns the number of errors. */
u64 orc_verify_sssp(u32 n, const u32* row, const u32* col, const u32* wt, u32 src, const u32* ref_dist,
                    const u32* dist, const u32* parent, u32 sample_paths, u64 seed, u64* report) {
    memset(report, 0, 6 * sizeof(u64));
    for (u32 v = 0; v < n; ++v) {
        report[0]++;
        if (dist[v] != ref_dist[v]) report[1]++;
    }
    for (u32 v = 0; v < n; ++v) {
        if (v == src || dist[v] == INF32) continue;
        report[2]++;
        u32 p = parent[v];
        int ok = p < n && dist[p] != INF32;
        if (ok) {
            ok = 0;
            for (u32 k = row[p]; k < row[p + 1]; ++k)
                if (col[k] == v && (u64)dist[p] + wt[k] == dist[v]) { ok = 1; break; }
        }
        if (!ok) report[3]++;
    }
    orc_rng r;
    rng_init(&r, seed);
    u32* path = (u32*)malloc(((size_t)n + 1) * sizeof(u32));
    for (u32 i = 0, tries = 0; i < sample_paths && tries < sample_paths * 50u; ++tries) {
        u32 t = rng_below(&r, n);
        if (ref_dist[t] == INF32) continue;
        ++i;
        report[4]++;
        u32 len = orc_reconstruct_path(parent, n, src, t, path, n + 1);
        if (!orc_validate_path(n, row, col, wt, path, len, src, t, ref_dist[t])) report[5]++;
    }
    free(path);
    return report[1] + report[3] + report[5];
}
