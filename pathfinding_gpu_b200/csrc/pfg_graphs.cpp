// pfg_graphs.cpp - host graph substrate: weight-sorted CSR builder, seeded
// generators of the benchmark workloads, DIMACS / SNAP / binary loaders.
// See include/pfg_graphs.h for the contracts.
#include "../../include/pfg_graphs.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <thread>
#include <vector>

typedef uint32_t u32;
typedef uint64_t u64;

struct pfg_graph {
    std::string name;
    u32 n = 0, m = 0;
    std::vector<u32> row, col, w;
    std::vector<double> x, y;
    pfg_graph_info info{};
};

// Message storage shared with the solver's C ABI (pfg_last_error).
extern "C" void pfg_internal_set_error(const char* msg);
static pfg_status gfail(pfg_status st, const std::string& msg) {
    pfg_internal_set_error(msg.c_str());
    return st;
}

namespace {

// SplitMix64 with the reference's seeding (include/common.h:44-56).
struct SplitMix {
    u64 s;
    explicit SplitMix(u64 seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x1234567ull) {}
    u64 next() {
        u64 z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
    u32 below(u32 n) { return (u32)(next() % n); }
};

// MurmurHash3 64-bit finaliser (used for weights of unweighted SNAP files,
// as the reference does, include/common.h:58-62).
inline u64 fmix64(u64 x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

template <class F>
void parallel_rows(u32 n, F&& fn) {
    unsigned T = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 65536 || T == 1) {
        fn(0u, n);
        return;
    }
    std::vector<std::thread> th;
    const u32 chunk = (n + T - 1) / T;
    for (unsigned t = 0; t < T; ++t) {
        const u32 b = t * chunk, e = std::min<u32>(n, b + chunk);
        if (b >= e) break;
        th.emplace_back([&fn, b, e] { fn(b, e); });
    }
    for (auto& x : th) x.join();
}

pfg_status build_csr(u32 n, const std::vector<u32>& src, const std::vector<u32>& dst,
                     const std::vector<u32>& win, std::vector<double>&& x, std::vector<double>&& y,
                     pfg_graph** out) {
    const u64 m_in = src.size();
    std::vector<u32> deg((size_t)n + 1, 0);
    u64 keep = 0;
    for (u64 i = 0; i < m_in; ++i) {
        if (src[i] >= n || dst[i] >= n) return gfail(PFG_ERR_INVALID_GRAPH, "arc endpoint out of range");
        if (src[i] != dst[i]) {
            deg[src[i]]++;
            keep++;
        }
    }
    if (keep >= 0xFFFFFFFFull)
        return gfail(PFG_ERR_INVALID_GRAPH, std::to_string(keep) +
                                                " arcs remain after dropping self loops; at most 2^32 - 2 fit the 32-bit row offsets");
    pfg_graph* g = new pfg_graph();
    g->n = n;
    g->m = (u32)keep;
    g->row.assign((size_t)n + 1, 0);
    for (u32 u = 0; u < n; ++u) g->row[u + 1] = g->row[u] + deg[u];
    g->col.resize(g->m);
    g->w.resize(g->m);
    {
        std::vector<u32> cursor(g->row.begin(), g->row.end() - 1);
        for (u64 i = 0; i < m_in; ++i) {
            const u32 s = src[i], d = dst[i];
            if (s == d) continue;
            const u32 pos = cursor[s]++;
            g->col[pos] = d;
            g->w[pos] = std::max<u32>(1u, win[i]);
        }
    }
    // Each row sorted by (w, dst).
    parallel_rows(n, [g](u32 b, u32 e) {
        std::vector<u64> tmp;
        for (u32 u = b; u < e; ++u) {
            const u32 r0 = g->row[u], r1 = g->row[u + 1];
            if (r1 - r0 < 2) continue;
            tmp.resize(r1 - r0);
            for (u32 k = r0; k < r1; ++k) tmp[k - r0] = ((u64)g->w[k] << 32) | g->col[k];
            std::sort(tmp.begin(), tmp.end());
            for (u32 k = r0; k < r1; ++k) {
                g->w[k] = (u32)(tmp[k - r0] >> 32);
                g->col[k] = (u32)tmp[k - r0];
            }
        }
    });
    pfg_graph_info& I = g->info;
    I.n = n;
    I.m = g->m;
    I.min_w = g->m ? 0xFFFFFFFFu : 0u;
    I.max_w = 0;
    double sum = 0.0;
    for (u32 k = 0; k < g->m; ++k) {
        I.min_w = std::min(I.min_w, g->w[k]);
        I.max_w = std::max(I.max_w, g->w[k]);
        sum += g->w[k];
    }
    I.avg_w = g->m ? sum / g->m : 0.0;
    I.max_deg = 0;
    for (u32 u = 0; u < n; ++u) I.max_deg = std::max(I.max_deg, g->row[u + 1] - g->row[u]);
    I.avg_deg = n ? (double)g->m / n : 0.0;
    g->x = std::move(x);
    g->y = std::move(y);
    I.has_xy = g->x.empty() ? 0 : 1;
    I.h_scale = 0.0;
    if (I.has_xy) {
        double scale = std::numeric_limits<double>::infinity();
        for (u32 u = 0; u < n; ++u)
            for (u32 k = g->row[u]; k < g->row[u + 1]; ++k) {
                const u32 v = g->col[k];
                const double dx = g->x[u] - g->x[v], dy = g->y[u] - g->y[v];
                const double e = std::sqrt(dx * dx + dy * dy);
                if (e > 1e-12) scale = std::min(scale, g->w[k] / e);
            }
        I.h_scale = std::isfinite(scale) ? scale : 0.0;
    }
    *out = g;
    return PFG_OK;
}

}  // namespace

// Wraps CSR arrays that are already in final form (built on the GPU by
// pfg_graph_from_edges_gpu) into a graph handle.
pfg_status pfg_internal_graph_from_csr(uint32_t n, std::vector<uint32_t>&& row, std::vector<uint32_t>&& col,
                                       std::vector<uint32_t>&& w, std::vector<double>&& x,
                                       std::vector<double>&& y, const pfg_graph_info& info, pfg_graph** out) {
    pfg_graph* g = new pfg_graph();
    g->n = n;
    g->m = info.m;
    g->row = std::move(row);
    g->col = std::move(col);
    g->w = std::move(w);
    g->x = std::move(x);
    g->y = std::move(y);
    g->info = info;
    *out = g;
    return PFG_OK;
}

namespace {

inline u32 grid_weight(SplitMix& rng) { return (u32)std::llround(100.0 * rng.uniform(1.0, 1.5)); }

}  // namespace

extern "C" pfg_status pfg_graph_from_edges(uint32_t n, uint64_t m_in, const uint32_t* src,
                                           const uint32_t* dst, const uint32_t* w, const double* x,
                                           const double* y, pfg_graph** out) {
    if (!out || (m_in && (!src || !dst || !w))) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((x == nullptr) != (y == nullptr)) return gfail(PFG_ERR_INVALID_ARGUMENT, "x and y must both be set");
    std::vector<u32> s(src, src + m_in), d(dst, dst + m_in), ww(w, w + m_in);
    std::vector<double> xs, ys;
    if (x) {
        xs.assign(x, x + n);
        ys.assign(y, y + n);
    }
    return build_csr(n, s, d, ww, std::move(xs), std::move(ys), out);
}

extern "C" pfg_status pfg_graph_gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, pfg_graph** out) {
    if (!out || rows == 0 || cols == 0 || (u64)rows * cols >= 0xFFFFFFFFull)
        return gfail(PFG_ERR_INVALID_ARGUMENT, "bad grid size");
    const u32 n = rows * cols;
    SplitMix rng(seed);
    std::vector<double> x(n), y(n);
    for (u32 r = 0; r < rows; ++r)
        for (u32 c = 0; c < cols; ++c) {
            x[(size_t)r * cols + c] = (double)c;
            y[(size_t)r * cols + c] = (double)r;
        }
    std::vector<u32> s, d, w;
    const size_t est = (size_t)n * 4;
    s.reserve(est);
    d.reserve(est);
    w.reserve(est);
    for (u32 r = 0; r < rows; ++r)
        for (u32 c = 0; c < cols; ++c) {
            const u32 id = r * cols + c;
            if (c + 1 < cols) {
                s.push_back(id); d.push_back(id + 1); w.push_back(grid_weight(rng));
                s.push_back(id + 1); d.push_back(id); w.push_back(grid_weight(rng));
            }
            if (r + 1 < rows) {
                s.push_back(id); d.push_back(id + cols); w.push_back(grid_weight(rng));
                s.push_back(id + cols); d.push_back(id); w.push_back(grid_weight(rng));
            }
        }
    pfg_status st = build_csr(n, s, d, w, std::move(x), std::move(y), out);
    if (st == PFG_OK) (*out)->name = "grid_" + std::to_string(rows) + "x" + std::to_string(cols);
    return st;
}

extern "C" pfg_status pfg_graph_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b,
                                         double c, uint32_t w_lo, uint32_t w_hi, uint64_t seed,
                                         pfg_graph** out) {
    if (!out || scale == 0 || scale > 30 || w_lo == 0 || w_hi < w_lo)
        return gfail(PFG_ERR_INVALID_ARGUMENT, "bad R-MAT parameters");
    const u32 n = 1u << scale;
    const u64 samples = (u64)n * edge_factor;
    SplitMix rng(seed);
    const double ab = a + b, abc = a + b + c;
    const u32 span = w_hi - w_lo + 1;
    // Sample arcs, bucket them by source (counting sort), then per row keep the
    // lightest copy of every (u, v).
    std::vector<u32> su, sv, sw;
    su.reserve(samples);
    sv.reserve(samples);
    sw.reserve(samples);
    for (u64 e = 0; e < samples; ++e) {
        u32 u = 0, v = 0;
        for (u32 bit = 0; bit < scale; ++bit) {
            const double r = rng.uniform();
            u32 bu = 0, bv = 0;
            if (r < a) {
            } else if (r < ab) {
                bv = 1;
            } else if (r < abc) {
                bu = 1;
            } else {
                bu = 1;
                bv = 1;
            }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        const u32 w = w_lo + rng.below(span);
        if (u == v) continue;
        su.push_back(u);
        sv.push_back(v);
        sw.push_back(w);
    }
    std::vector<u32> start((size_t)n + 1, 0);
    for (u32 u : su) start[u + 1]++;
    for (u32 i = 0; i < n; ++i) start[i + 1] += start[i];
    std::vector<u64> packed(su.size());
    {
        std::vector<u32> cur(start.begin(), start.end() - 1);
        for (size_t i = 0; i < su.size(); ++i) packed[cur[su[i]]++] = ((u64)sv[i] << 32) | sw[i];
    }
    std::vector<u32>().swap(su);
    std::vector<u32>().swap(sv);
    std::vector<u32>().swap(sw);
    std::vector<u32> keep_cnt(n, 0);
    parallel_rows(n, [&](u32 b0, u32 e0) {
        for (u32 u = b0; u < e0; ++u) {
            u64* p = packed.data() + start[u];
            const u32 len = start[u + 1] - start[u];
            std::sort(p, p + len);  // by (v, w): first copy of each v is the lightest
            u32 k = 0;
            for (u32 i = 0; i < len; ++i)
                if (k == 0 || (p[i] >> 32) != (p[k - 1] >> 32)) p[k++] = p[i];
            keep_cnt[u] = k;
        }
    });
    std::vector<u32> s, d, w;
    u64 total = 0;
    for (u32 u = 0; u < n; ++u) total += keep_cnt[u];
    s.reserve(total);
    d.reserve(total);
    w.reserve(total);
    for (u32 u = 0; u < n; ++u) {
        const u64* p = packed.data() + start[u];
        for (u32 i = 0; i < keep_cnt[u]; ++i) {
            s.push_back(u);
            d.push_back((u32)(p[i] >> 32));
            w.push_back((u32)p[i]);
        }
    }
    std::vector<u64>().swap(packed);
    pfg_status st = build_csr(n, s, d, w, {}, {}, out);
    if (st == PFG_OK) (*out)->name = "rmat_s" + std::to_string(scale) + "_ef" + std::to_string(edge_factor);
    return st;
}

extern "C" pfg_status pfg_graph_gen_road(uint32_t side, double removal, double shortcut,
                                         uint32_t radius, double factor, uint64_t seed,
                                         pfg_graph** out) {
    if (!out || side < 2 || (u64)side * side >= 0xFFFFFFFFull)
        return gfail(PFG_ERR_INVALID_ARGUMENT, "bad road grid size");
    const u32 n = side * side;
    SplitMix rng(seed);
    std::vector<double> x(n), y(n);
    for (u32 r = 0; r < side; ++r)
        for (u32 c = 0; c < side; ++c) {
            x[(size_t)r * side + c] = (double)c;
            y[(size_t)r * side + c] = (double)r;
        }
    std::vector<u32> s, d, w;
    s.reserve((size_t)n * 4);
    d.reserve((size_t)n * 4);
    w.reserve((size_t)n * 4);
    auto add_pair = [&](u32 a, u32 b) {
        s.push_back(a); d.push_back(b); w.push_back(grid_weight(rng));
        s.push_back(b); d.push_back(a); w.push_back(grid_weight(rng));
    };
    for (u32 r = 0; r < side; ++r)
        for (u32 c = 0; c < side; ++c) {
            const u32 id = r * side + c;
            if (c + 1 < side && !(rng.uniform() < removal)) add_pair(id, id + 1);
            if (r + 1 < side && !(rng.uniform() < removal)) add_pair(id, id + side);
        }
    const int R = (int)radius;
    for (u32 v = 0; v < n; ++v) {
        if (!(rng.uniform() < shortcut)) continue;
        const int r = (int)(v / side), c = (int)(v % side);
        const int r0 = std::max(0, r - R), r1 = std::min((int)side - 1, r + R);
        const int c0 = std::max(0, c - R), c1 = std::min((int)side - 1, c + R);
        u32 t = v;
        for (int tries = 0; tries < 16 && t == v; ++tries) {
            const int tr = r0 + (int)rng.below((u32)(r1 - r0 + 1));
            const int tc = c0 + (int)rng.below((u32)(c1 - c0 + 1));
            t = (u32)tr * side + (u32)tc;
        }
        if (t == v) continue;
        const double dx = x[v] - x[t], dy = y[v] - y[t];
        const u32 wt = (u32)std::ceil(factor * 100.0 * std::sqrt(dx * dx + dy * dy));
        s.push_back(v); d.push_back(t); w.push_back(wt);
        s.push_back(t); d.push_back(v); w.push_back(wt);
    }
    pfg_status st = build_csr(n, s, d, w, std::move(x), std::move(y), out);
    if (st == PFG_OK) (*out)->name = "road_" + std::to_string(side) + "x" + std::to_string(side);
    return st;
}

extern "C" pfg_status pfg_graph_union(const pfg_graph* const* parts, uint32_t count, pfg_graph** out) {
    if (!out || !parts || count == 0) return gfail(PFG_ERR_INVALID_ARGUMENT, "no graphs to join");
    u64 n = 0, m = 0;
    bool xy = true;
    for (u32 i = 0; i < count; ++i) {
        if (!parts[i]) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL graph");
        n += parts[i]->n;
        m += parts[i]->m;
        xy = xy && !parts[i]->x.empty();
    }
    if (n >= 0xFFFFFFFFull || m >= 0xFFFFFFFFull) return gfail(PFG_ERR_INVALID_GRAPH, "union too large");
    std::vector<u32> s, d, w;
    s.reserve(m);
    d.reserve(m);
    w.reserve(m);
    std::vector<double> x, y;
    u32 base = 0;
    for (u32 i = 0; i < count; ++i) {
        const pfg_graph* g = parts[i];
        for (u32 u = 0; u < g->n; ++u)
            for (u32 k = g->row[u]; k < g->row[u + 1]; ++k) {
                s.push_back(base + u);
                d.push_back(base + g->col[k]);
                w.push_back(g->w[k]);
            }
        if (xy) {
            x.insert(x.end(), g->x.begin(), g->x.end());
            y.insert(y.end(), g->y.begin(), g->y.end());
        }
        base += g->n;
    }
    return build_csr((u32)n, s, d, w, std::move(x), std::move(y), out);
}

// ---------------------------------------------------------------------------
// Loaders
// ---------------------------------------------------------------------------
namespace {
bool read_file(const char* path, std::string& buf) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    f.seekg(0, std::ios::end);
    const std::streamoff sz = f.tellg();
    f.seekg(0, std::ios::beg);
    buf.resize((size_t)std::max<std::streamoff>(0, sz));
    if (sz > 0) f.read(&buf[0], sz);
    return (bool)f || f.eof();
}
inline void skip_blank(const char*& p, const char* e) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
}
inline void next_line(const char*& p, const char* e) {
    while (p < e && *p != '\n') ++p;
    if (p < e) ++p;
}
inline bool read_int(const char*& p, const char* e, long long& out) {
    skip_blank(p, e);
    bool neg = false;
    if (p < e && (*p == '-' || *p == '+')) neg = *p++ == '-';
    if (p >= e || *p < '0' || *p > '9') return false;
    long long v = 0;
    while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
    out = neg ? -v : v;
    return true;
}
std::string base_name(const char* path) {
    std::string s(path);
    const size_t k = s.find_last_of("/\\");
    return k == std::string::npos ? s : s.substr(k + 1);
}
}  // namespace

extern "C" pfg_status pfg_graph_load_dimacs(const char* gr_path, const char* co_path, pfg_graph** out) {
    if (!gr_path || !out) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::string buf;
    if (!read_file(gr_path, buf)) return gfail(PFG_ERR_INVALID_ARGUMENT, std::string("cannot open ") + gr_path);
    const char* p = buf.data();
    const char* e = p + buf.size();
    long long n = -1;
    std::vector<u32> s, d, w;
    while (p < e) {
        if (*p == 'p') {  // p sp <n> <m>
            ++p;
            skip_blank(p, e);
            while (p < e && *p != ' ' && *p != '\t') ++p;
            long long nn = 0, mm = 0;
            read_int(p, e, nn);
            read_int(p, e, mm);
            n = nn;
            if (mm > 0) {
                s.reserve((size_t)mm);
                d.reserve((size_t)mm);
                w.reserve((size_t)mm);
            }
        } else if (*p == 'a') {  // a <u> <v> <w>, 1-based
            ++p;
            long long u, v, ww;
            if (read_int(p, e, u) && read_int(p, e, v) && read_int(p, e, ww)) {
                if (u < 1 || v < 1 || ww < 0) return gfail(PFG_ERR_INVALID_GRAPH, "bad DIMACS arc line");
                s.push_back((u32)(u - 1));
                d.push_back((u32)(v - 1));
                w.push_back((u32)ww);
            }
        }
        next_line(p, e);
    }
    if (n <= 0 || n >= 0xFFFFFFFFll) return gfail(PFG_ERR_INVALID_GRAPH, "Invalid DIMACS .gr (missing 'p sp' line)");
    for (size_t i = 0; i < s.size(); ++i)
        if (s[i] >= (u64)n || d[i] >= (u64)n) return gfail(PFG_ERR_INVALID_GRAPH, "DIMACS arc endpoint > n");
    std::vector<double> x, y;
    if (co_path && *co_path) {
        std::string cb;
        if (!read_file(co_path, cb)) return gfail(PFG_ERR_INVALID_ARGUMENT, std::string("cannot open ") + co_path);
        std::vector<double> lon((size_t)n, 0.0), lat((size_t)n, 0.0);
        const char* q = cb.data();
        const char* qe = q + cb.size();
        double lat_sum = 0.0;
        u64 cnt = 0;
        while (q < qe) {
            if (*q == 'v') {  // v <id> <lon * 1e6> <lat * 1e6>
                ++q;
                long long id, X, Y;
                if (read_int(q, qe, id) && read_int(q, qe, X) && read_int(q, qe, Y) && id >= 1 && id <= n) {
                    lon[(size_t)id - 1] = (double)X;
                    lat[(size_t)id - 1] = (double)Y;
                    lat_sum += (double)Y;
                    cnt++;
                }
            }
            next_line(q, qe);
        }
        // Equirectangular projection around the mean latitude, as the reference
        // does (src/graph.cpp:270-279), so hScale calibrates the units.
        const double lat0 = cnt ? (lat_sum / cnt) * 1e-6 * 3.14159265358979323846 / 180.0 : 0.0;
        const double cs = std::cos(lat0);
        x.resize((size_t)n);
        y.resize((size_t)n);
        for (size_t i = 0; i < (size_t)n; ++i) {
            x[i] = lon[i] * cs;
            y[i] = lat[i];
        }
    }
    pfg_status st = build_csr((u32)n, s, d, w, std::move(x), std::move(y), out);
    if (st == PFG_OK) (*out)->name = base_name(gr_path);
    return st;
}

extern "C" pfg_status pfg_graph_load_snap(const char* path, int32_t symmetrize, uint32_t max_w,
                                          uint64_t seed, pfg_graph** out) {
    if (!path || !out || max_w == 0) return gfail(PFG_ERR_INVALID_ARGUMENT, "bad argument");
    std::string buf;
    if (!read_file(path, buf)) return gfail(PFG_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    const char* p = buf.data();
    const char* e = p + buf.size();
    std::vector<u32> s, d, w;
    u64 max_id = 0;
    bool any = false;
    while (p < e) {
        skip_blank(p, e);
        if (p >= e) break;
        if (*p == '#' || *p == '%' || *p == '\n') {
            next_line(p, e);
            continue;
        }
        long long u, v, ww = -1;
        if (!read_int(p, e, u) || !read_int(p, e, v)) {
            next_line(p, e);
            continue;
        }
        const char* save = p;
        if (!read_int(p, e, ww)) {
            p = save;
            ww = -1;
        }
        next_line(p, e);
        if (u < 0 || v < 0 || u >= 0xFFFFFFFFll || v >= 0xFFFFFFFFll) continue;
        if (ww <= 0) {  // unweighted: symmetric, reproducible weight
            const u64 lo = (u64)std::min(u, v), hi = (u64)std::max(u, v);
            ww = 1 + (long long)(fmix64(((lo << 32) | hi) ^ seed) % max_w);
        }
        s.push_back((u32)u);
        d.push_back((u32)v);
        w.push_back((u32)std::min<long long>(ww, 0xFFFFFFFEll));
        if (symmetrize) {
            s.push_back((u32)v);
            d.push_back((u32)u);
            w.push_back((u32)std::min<long long>(ww, 0xFFFFFFFEll));
        }
        max_id = std::max<u64>(max_id, (u64)std::max(u, v));
        any = true;
    }
    if (!any) return gfail(PFG_ERR_INVALID_GRAPH, "SNAP file has no arcs");
    if (max_id + 1 >= 0xFFFFFFFFull) return gfail(PFG_ERR_INVALID_GRAPH, "vertex id too large");
    pfg_status st = build_csr((u32)(max_id + 1), s, d, w, {}, {}, out);
    if (st == PFG_OK) (*out)->name = base_name(path);
    return st;
}

static const char kMagic[8] = {'P', 'F', 'C', 'S', 'R', '0', '0', '1'};

extern "C" pfg_status pfg_graph_save_binary(const pfg_graph* g, const char* path) {
    if (!g || !path) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE* f = fopen(path, "wb");
    if (!f) return gfail(PFG_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
    const u32 name_len = (u32)g->name.size(), has_xy = g->x.empty() ? 0u : 1u;
    bool ok = fwrite(kMagic, 1, 8, f) == 8;
    ok = ok && fwrite(&g->n, 4, 1, f) == 1 && fwrite(&g->m, 4, 1, f) == 1;
    ok = ok && fwrite(&has_xy, 4, 1, f) == 1 && fwrite(&name_len, 4, 1, f) == 1;
    ok = ok && fwrite(g->name.data(), 1, name_len, f) == name_len;
    ok = ok && fwrite(g->row.data(), 4, (size_t)g->n + 1, f) == (size_t)g->n + 1;
    ok = ok && fwrite(g->col.data(), 4, g->m, f) == g->m;
    ok = ok && fwrite(g->w.data(), 4, g->m, f) == g->m;
    if (has_xy) {
        ok = ok && fwrite(g->x.data(), 8, g->n, f) == g->n;
        ok = ok && fwrite(g->y.data(), 8, g->n, f) == g->n;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? PFG_OK : gfail(PFG_ERR_INVALID_ARGUMENT, "write failed");
}

extern "C" pfg_status pfg_graph_load_binary(const char* path, pfg_graph** out) {
    if (!path || !out) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE* f = fopen(path, "rb");
    if (!f) return gfail(PFG_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    char mg[8];
    u32 n = 0, m = 0, has_xy = 0, name_len = 0;
    bool ok = fread(mg, 1, 8, f) == 8 && memcmp(mg, kMagic, 8) == 0;
    ok = ok && fread(&n, 4, 1, f) == 1 && fread(&m, 4, 1, f) == 1 && fread(&has_xy, 4, 1, f) == 1 &&
         fread(&name_len, 4, 1, f) == 1 && name_len < (1u << 20);
    std::string name(ok ? name_len : 0, '\0');
    if (ok && name_len) ok = fread(&name[0], 1, name_len, f) == name_len;
    std::vector<u32> ro, ci, w;
    std::vector<double> x, y;
    if (ok) {
        ro.resize((size_t)n + 1);
        ci.resize(m);
        w.resize(m);
        ok = fread(ro.data(), 4, ro.size(), f) == ro.size() && fread(ci.data(), 4, m, f) == m &&
             fread(w.data(), 4, m, f) == m;
    }
    if (ok && has_xy) {
        x.resize(n);
        y.resize(n);
        ok = fread(x.data(), 8, n, f) == n && fread(y.data(), 8, n, f) == n;
    }
    fclose(f);
    if (!ok) return gfail(PFG_ERR_INVALID_GRAPH, std::string("not a PFCSR001 file: ") + path);
    if (ro[0] != 0 || ro[n] != m) return gfail(PFG_ERR_INVALID_GRAPH, "corrupt row offsets");
    // Rebuilt through the CSR builder so statistics and hScale are recomputed
    // (the reference does the same, src/graph.cpp:358-366).
    std::vector<u32> src(m);
    for (u32 u = 0; u < n; ++u) {
        if (ro[u + 1] < ro[u] || ro[u + 1] > m) return gfail(PFG_ERR_INVALID_GRAPH, "corrupt row offsets");
        for (u32 k = ro[u]; k < ro[u + 1]; ++k) src[k] = u;
    }
    pfg_status st = build_csr(n, src, ci, w, std::move(x), std::move(y), out);
    if (st == PFG_OK) (*out)->name = name;
    return st;
}

extern "C" pfg_status pfg_graph_get_info(const pfg_graph* g, pfg_graph_info* out) {
    if (!g || !out) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = g->info;
    return PFG_OK;
}
extern "C" const uint32_t* pfg_graph_row_offsets(const pfg_graph* g) { return g ? g->row.data() : nullptr; }
extern "C" const uint32_t* pfg_graph_col_indices(const pfg_graph* g) { return g ? g->col.data() : nullptr; }
extern "C" const uint32_t* pfg_graph_weights(const pfg_graph* g) { return g ? g->w.data() : nullptr; }
extern "C" const double* pfg_graph_x(const pfg_graph* g) { return g && !g->x.empty() ? g->x.data() : nullptr; }
extern "C" const double* pfg_graph_y(const pfg_graph* g) { return g && !g->y.empty() ? g->y.data() : nullptr; }
extern "C" void pfg_graph_free(pfg_graph* g) { delete g; }

extern "C" pfg_status pfg_graph_pick_sources(const pfg_graph* g, uint32_t count, uint64_t seed,
                                             uint32_t* out) {
    if (!g || (count && !out)) return gfail(PFG_ERR_INVALID_ARGUMENT, "NULL argument");
    SplitMix rng(seed);
    u32 got = 0;
    for (u64 tries = 0; got < count && tries < (u64)count * 1000u + 1000u; ++tries) {
        const u32 v = rng.below(g->n);
        if (g->row[v + 1] > g->row[v]) out[got++] = v;
    }
    while (got < count) out[got++] = 0;
    return PFG_OK;
}
