// pfg_csr.cu - CSR construction on the GPU.
//
// Same result, word for word, as the reference's buildCSR (src/graph.cpp:23-104)
// and the host builder in pfg_graphs.cpp: self loops dropped, weights below 1
// raised to 1, arcs grouped by source, every row sorted by (w, dst), then the
// graph statistics (min / max / mean weight, max degree, mean degree) and the
// A* scale h_scale = min over arcs of w / |p(u) - p(v)| (arcs with a length
// above 1e-12).
//
//   1. degree count (one atomicAdd per kept arc) and endpoint check
//   2. exclusive scan of the degrees into row offsets (block scans + one pass
//      over the block totals + offset add)
//   3. scatter: each kept arc writes the 64-bit key (w << 32) | dst at an
//      atomically reserved position of its row. The order inside a row is
//      arbitrary here; the next step makes it canonical because (w, dst) is a
//      total order (equal keys are equal arcs).
//   4. segmented sort of the keys, by row length: rows of up to 32 arcs by one
//      thread (insertion sort), up to 2048 by one CTA (bitonic sort in shared
//      memory), longer rows (R-MAT hubs) by one CTA: bitonic sort of 2048-key
//      chunks, then merge-path merges of neighbouring runs, ping-ponging with
//      a scratch array
//   5. split keys into col / w; statistics with explicitly rounded double
//      arithmetic (no contraction), so h_scale matches the host exactly.
#include "../../include/pfg.h"
#include "../../include/pfg_graphs.h"
#include "pfg_common.cuh"
#include "pfg_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

using namespace pfg;

namespace {

constexpr u32 SCAN_B = 1024;   // elements per block of the scan
constexpr u32 MID_MAX = 2048;  // longest row sorted in one shared-memory pass
constexpr u32 SORT_BS = 256;   // threads of the CTA sorts

__global__ void k_count(u64 m_in, const u32* __restrict__ src, const u32* __restrict__ dst, u32 n,
                        u32* __restrict__ deg, unsigned long long* kept, u32* bad) {
    u32 local = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < m_in; i += (u64)gridDim.x * blockDim.x) {
        const u32 s = src[i], d = dst[i];
        if (s >= n || d >= n) {
            atomicOr(bad, 1u);
            continue;
        }
        if (s != d) {
            atomicAdd(deg + s, 1u);
            ++local;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
    if ((threadIdx.x & 31u) == 0 && local) atomicAdd(kept, (unsigned long long)local);
}

// Exclusive scan inside a block of SCAN_B elements (blockDim = SCAN_B); the
// block total goes to bsum[blockIdx.x].
__device__ __forceinline__ u32 block_scan_excl(u32 v, u32& total) {
    __shared__ u32 warp_tot[32];
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    u32 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (u32)o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        u32 t = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= (u32)o) t += y;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[31];
    const u32 base = warp ? warp_tot[warp - 1] : 0u;
    __syncthreads();
    return base + x - v;
}

__global__ void k_scan_blocks(const u32* __restrict__ in, u32 n, u32* __restrict__ out, u32* __restrict__ bsum) {
    const u32 i = blockIdx.x * SCAN_B + threadIdx.x;
    u32 total = 0;
    const u32 e = block_scan_excl(i < n ? in[i] : 0u, total);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// One block: exclusive scan of the nb block totals in place, chunk by chunk;
// the grand total goes to *total.
__global__ void k_scan_sums(u32* bsum, u32 nb, u32* total_out) {
    __shared__ u32 carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (u32 b = 0; b < nb; b += SCAN_B) {
        const u32 i = b + threadIdx.x;
        u32 t = 0;
        const u32 e = block_scan_excl(i < nb ? bsum[i] : 0u, t);
        const u32 c = carry;
        if (i < nb) bsum[i] = c + e;
        __syncthreads();
        if (threadIdx.x == 0) carry = c + t;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(u32* out, u32 n, const u32* bsum) {
    const u32 i = blockIdx.x * SCAN_B + threadIdx.x;
    if (i < n) out[i] += bsum[blockIdx.x];
}

__global__ void k_scatter(u64 m_in, const u32* __restrict__ src, const u32* __restrict__ dst,
                          const u32* __restrict__ w, u32* __restrict__ cursor, u64* __restrict__ key) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < m_in; i += (u64)gridDim.x * blockDim.x) {
        const u32 s = src[i], d = dst[i];
        if (s == d) continue;
        const u32 wi = w[i] < 1u ? 1u : w[i];
        const u32 pos = atomicAdd(cursor + s, 1u);
        key[pos] = ((u64)wi << 32) | d;
    }
}

// Rows of 2..32 arcs: insertion sort by one thread. Longer rows are listed
// for the CTA sorts.
__global__ void k_sort_small(const u32* __restrict__ row, u32 n, u64* __restrict__ key, u32* mid_list,
                             u32* mid_cnt, u32* big_list, u32* big_cnt) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const u32 r0 = row[u], r1 = row[u + 1], len = r1 - r0;
        if (len < 2) continue;
        if (len > MID_MAX) {
            big_list[atomicAdd(big_cnt, 1u)] = u;
        } else if (len > 32) {
            mid_list[atomicAdd(mid_cnt, 1u)] = u;
        } else {
            u64 a[32];
            for (u32 i = 0; i < len; ++i) {
                const u64 k = key[r0 + i];
                u32 j = i;
                while (j > 0 && a[j - 1] > k) {
                    a[j] = a[j - 1];
                    --j;
                }
                a[j] = k;
            }
            for (u32 i = 0; i < len; ++i) key[r0 + i] = a[i];
        }
    }
}

// Bitonic sort of sh[0..P) (P a power of two <= MID_MAX) by the whole CTA.
__device__ void bitonic_sort_shared(u64* sh, u32 P) {
    for (u32 k = 2; k <= P; k <<= 1) {
        for (u32 j = k >> 1; j > 0; j >>= 1) {
            for (u32 i = threadIdx.x; i < P; i += blockDim.x) {
                const u32 ixj = i ^ j;
                if (ixj > i) {
                    const u64 a = sh[i], b = sh[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        sh[i] = b;
                        sh[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Sorts key[b, b + len) (len <= MID_MAX) in shared memory.
__device__ void sort_run_shared(u64* __restrict__ key, u32 b, u32 len, u64* sh) {
    u32 P = 1;
    while (P < len) P <<= 1;
    for (u32 i = threadIdx.x; i < P; i += blockDim.x) sh[i] = i < len ? key[b + i] : ~0ull;
    __syncthreads();
    bitonic_sort_shared(sh, P);
    for (u32 i = threadIdx.x; i < len; i += blockDim.x) key[b + i] = sh[i];
    __syncthreads();
}

__global__ void k_sort_mid(const u32* __restrict__ row, u64* __restrict__ key, const u32* list, const u32* cnt) {
    __shared__ u64 sh[MID_MAX];
    const u32 c = *cnt;
    for (u32 i = blockIdx.x; i < c; i += gridDim.x) {
        const u32 u = list[i];
        sort_run_shared(key, row[u], row[u + 1] - row[u], sh);
    }
}

// Merges the sorted runs A = in[a0, a0 + la) and B = in[b0, b0 + lb) into
// out[o0, o0 + la + lb) with the whole CTA (merge path: each thread finds its
// diagonal's split by binary search and merges its share).
__device__ void merge_runs(const u64* __restrict__ in, u64* __restrict__ out, u32 a0, u32 la, u32 b0, u32 lb,
                           u32 o0) {
    const u32 total = la + lb;
    const u32 per = (total + blockDim.x - 1) / blockDim.x;
    const u32 d0 = min(total, threadIdx.x * per), d1 = min(total, d0 + per);
    if (d0 >= d1) return;
    // split of diagonal d0: i elements from A, d0 - i from B
    u32 lo = d0 > lb ? d0 - lb : 0u, hi = min(d0, la);
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (in[a0 + mid] <= in[b0 + d0 - 1 - mid]) lo = mid + 1; else hi = mid;
    }
    u32 i = lo, j = d0 - lo;
    for (u32 d = d0; d < d1; ++d) {
        const bool take_a = j >= lb || (i < la && in[a0 + i] <= in[b0 + j]);
        out[o0 + d] = take_a ? in[a0 + i++] : in[b0 + j++];
    }
}

__global__ void k_sort_big(const u32* __restrict__ row, u64* __restrict__ key, u64* __restrict__ tmp,
                           const u32* list, const u32* cnt) {
    __shared__ u64 sh[MID_MAX];
    const u32 c = *cnt;
    for (u32 it = blockIdx.x; it < c; it += gridDim.x) {
        const u32 u = list[it];
        const u32 r0 = row[u], len = row[u + 1] - r0;
        for (u32 b = 0; b < len; b += MID_MAX) sort_run_shared(key, r0 + b, min(MID_MAX, len - b), sh);
        u64* src = key;
        u64* dst = tmp;
        for (u32 wdt = MID_MAX; wdt < len; wdt <<= 1) {
            for (u32 s = 0; s < len; s += 2 * wdt) {
                const u32 la = min(wdt, len - s);
                const u32 lb = s + wdt < len ? min(wdt, len - s - wdt) : 0u;
                merge_runs(src, dst, r0 + s, la, r0 + s + la, lb, r0 + s);
            }
            __syncthreads();
            u64* t = src;
            src = dst;
            dst = t;
        }
        if (src != key) {
            for (u32 i = threadIdx.x; i < len; i += blockDim.x) key[r0 + i] = src[r0 + i];
        }
        __syncthreads();
    }
}

__global__ void k_split(u64 m, const u64* __restrict__ key, u32* __restrict__ col, u32* __restrict__ w) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x) {
        const u64 k = key[i];
        col[i] = (u32)k;
        w[i] = (u32)(k >> 32);
    }
}

struct StatsOut {
    u32 min_w, max_w, max_deg, pad;
    unsigned long long sum_w;
    unsigned long long hs_bits;  // bits of the smallest positive w / length (+inf if none)
};

__global__ void k_stats(const u32* __restrict__ row, u32 n, const u32* __restrict__ col, const u32* __restrict__ w,
                        const double* __restrict__ x, const double* __restrict__ y, StatsOut* out) {
    u32 mn = 0xFFFFFFFFu, mx = 0, md = 0;
    unsigned long long sum = 0;
    double hs = __longlong_as_double(0x7FF0000000000000ll);
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const u32 r0 = row[u], r1 = row[u + 1];
        md = max(md, r1 - r0);
        for (u32 k = r0; k < r1; ++k) {
            const u32 wk = w[k];
            mn = min(mn, wk);
            mx = max(mx, wk);
            sum += wk;
            if (x) {
                const u32 v = col[k];
                const double dx = __dsub_rn(x[u], x[v]), dy = __dsub_rn(y[u], y[v]);
                const double e = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
                if (e > 1e-12) {
                    const double q = __ddiv_rn((double)wk, e);
                    hs = q < hs ? q : hs;
                }
            }
        }
    }
    atomicMin(&out->min_w, mn);
    atomicMax(&out->max_w, mx);
    atomicMax(&out->max_deg, md);
    if (sum) atomicAdd(&out->sum_w, sum);
    // positive doubles order like their bit patterns
    atomicMin(&out->hs_bits, (unsigned long long)__double_as_longlong(hs));
}

struct DevBuf {
    std::vector<void*> p;
    template <class T>
    cudaError_t alloc(T** q, size_t count) {
        void* v = nullptr;
        const cudaError_t e = cudaMalloc(&v, std::max<size_t>(1, count) * sizeof(T));
        if (e == cudaSuccess) p.push_back(v);
        *q = (T*)v;
        return e;
    }
    ~DevBuf() {
        for (void* v : p) cudaFree(v);
    }
};

#define C_CUDA(call)                                                                            \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess) {                                                               \
            cudaGetLastError();                                                                 \
            return set_error(e__ == cudaErrorMemoryAllocation ? PFG_ERR_OUT_OF_MEMORY : PFG_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e__));                  \
        }                                                                                       \
    } while (0)

}  // namespace

extern "C" pfg_status pfg_csr_build_device(uint32_t n, uint64_t m_in, const uint32_t* d_src, const uint32_t* d_dst,
                                           const uint32_t* d_w, const double* d_x, const double* d_y,
                                           uint32_t* d_row, uint32_t* d_col, uint32_t* d_w_out,
                                           pfg_graph_info* info, int32_t device, void* stream) {
    if (n == 0 || !d_row || !info || (m_in && (!d_src || !d_dst || !d_w || !d_col || !d_w_out)))
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_csr_build_device: bad argument");
    if ((d_x == nullptr) != (d_y == nullptr))
        return set_error(PFG_ERR_INVALID_ARGUMENT, "x and y must both be set or both be NULL");
    if (n == 0xFFFFFFFFu) return set_error(PFG_ERR_INVALID_ARGUMENT, "n must be < 2^32 - 1");
    C_CUDA(cudaSetDevice(device));
    cudaStream_t st = (cudaStream_t)stream;
    int sms = 1;
    C_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    DevBuf buf;
    u32 *deg = nullptr, *bsum = nullptr, *cursor = nullptr, *lists = nullptr, *flags = nullptr;
    u64* key = nullptr;
    unsigned long long* kept = nullptr;
    StatsOut* so = nullptr;
    const u32 nb = (n + SCAN_B - 1) / SCAN_B;
    C_CUDA(buf.alloc(&deg, (size_t)n));
    C_CUDA(buf.alloc(&bsum, (size_t)nb));
    C_CUDA(buf.alloc(&cursor, (size_t)n));
    C_CUDA(buf.alloc(&lists, 2 * (size_t)n));
    C_CUDA(buf.alloc(&flags, 8));  // bad, total, mid count, big count
    C_CUDA(buf.alloc(&kept, 1));
    C_CUDA(buf.alloc(&so, 1));
    C_CUDA(buf.alloc(&key, (size_t)m_in));
    C_CUDA(cudaMemsetAsync(deg, 0, (size_t)n * 4, st));
    C_CUDA(cudaMemsetAsync(flags, 0, 8 * 4, st));
    C_CUDA(cudaMemsetAsync(kept, 0, 8, st));
    const u32 grid_arcs = (u32)std::max<u64>(1, std::min<u64>((m_in + 255) / 256, (u64)sms * 16));
    const u32 grid_rows = (u32)std::max<u64>(1, std::min<u64>(((u64)n + 255) / 256, (u64)sms * 16));
    if (m_in) k_count<<<grid_arcs, 256, 0, st>>>(m_in, d_src, d_dst, n, deg, kept, flags);
    C_CUDA(cudaGetLastError());
    u32 h_flags[2] = {0, 0};
    unsigned long long h_kept = 0;
    C_CUDA(cudaMemcpyAsync(h_flags, flags, 4, cudaMemcpyDeviceToHost, st));
    C_CUDA(cudaMemcpyAsync(&h_kept, kept, 8, cudaMemcpyDeviceToHost, st));
    C_CUDA(cudaStreamSynchronize(st));
    if (h_flags[0]) return set_error(PFG_ERR_INVALID_GRAPH, "arc endpoint out of range");
    if (h_kept >= 0xFFFFFFFFull) return set_error(PFG_ERR_INVALID_GRAPH, "%llu arcs remain after dropping self loops; at most 2^32 - 2 fit the 32-bit row offsets", (unsigned long long)h_kept);
    const u32 m = (u32)h_kept;

    k_scan_blocks<<<nb, SCAN_B, 0, st>>>(deg, n, d_row, bsum);
    k_scan_sums<<<1, SCAN_B, 0, st>>>(bsum, nb, d_row + n);
    k_scan_add<<<nb, SCAN_B, 0, st>>>(d_row, n, bsum);
    C_CUDA(cudaGetLastError());
    C_CUDA(cudaMemcpyAsync(cursor, d_row, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
    if (m_in) k_scatter<<<grid_arcs, 256, 0, st>>>(m_in, d_src, d_dst, d_w, cursor, key);
    k_sort_small<<<grid_rows, 256, 0, st>>>(d_row, n, key, lists, flags + 2, lists + n, flags + 3);
    k_sort_mid<<<sms * 4, SORT_BS, 0, st>>>(d_row, key, lists, flags + 2);
    C_CUDA(cudaGetLastError());
    u32 h_big = 0;
    C_CUDA(cudaMemcpyAsync(&h_big, flags + 3, 4, cudaMemcpyDeviceToHost, st));
    C_CUDA(cudaStreamSynchronize(st));
    if (h_big) {
        u64* tmp = nullptr;
        C_CUDA(buf.alloc(&tmp, (size_t)m));
        k_sort_big<<<std::min<u32>(h_big, (u32)sms * 2), SORT_BS, 0, st>>>(d_row, key, tmp, lists + n, flags + 3);
        C_CUDA(cudaGetLastError());
        C_CUDA(cudaStreamSynchronize(st));  // tmp is freed on return
    }
    if (m) k_split<<<grid_arcs, 256, 0, st>>>(m, key, d_col, d_w_out);
    StatsOut s0;
    memset(&s0, 0, sizeof(s0));
    s0.min_w = 0xFFFFFFFFu;
    s0.hs_bits = 0x7FF0000000000000ull;
    C_CUDA(cudaMemcpyAsync(so, &s0, sizeof(s0), cudaMemcpyHostToDevice, st));
    k_stats<<<grid_rows, 256, 0, st>>>(d_row, n, d_col, d_w_out, d_x, d_y, so);
    C_CUDA(cudaGetLastError());
    StatsOut hs;
    C_CUDA(cudaMemcpyAsync(&hs, so, sizeof(hs), cudaMemcpyDeviceToHost, st));
    C_CUDA(cudaStreamSynchronize(st));
    memset(info, 0, sizeof(*info));
    info->n = n;
    info->m = m;
    info->min_w = m ? hs.min_w : 0u;
    info->max_w = hs.max_w;
    info->max_deg = hs.max_deg;
    info->has_xy = d_x ? 1 : 0;
    info->avg_w = m ? (double)hs.sum_w / m : 0.0;
    info->avg_deg = (double)m / n;
    double scale;
    memcpy(&scale, &hs.hs_bits, 8);
    info->h_scale = (d_x && std::isfinite(scale)) ? scale : 0.0;
    return PFG_OK;
}

// Defined in pfg_graphs.cpp: wraps finished CSR arrays into a graph handle.
pfg_status pfg_internal_graph_from_csr(uint32_t n, std::vector<uint32_t>&& row, std::vector<uint32_t>&& col,
                                       std::vector<uint32_t>&& w, std::vector<double>&& x,
                                       std::vector<double>&& y, const pfg_graph_info& info, pfg_graph** out);

extern "C" pfg_status pfg_graph_from_edges_gpu(uint32_t n, uint64_t m_in, const uint32_t* src, const uint32_t* dst,
                                               const uint32_t* w, const double* x, const double* y, int32_t device,
                                               pfg_graph** out) {
    if (!out || n == 0 || (m_in && (!src || !dst || !w)))
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_graph_from_edges_gpu: bad argument");
    if ((x == nullptr) != (y == nullptr)) return set_error(PFG_ERR_INVALID_ARGUMENT, "x and y must both be set");
    *out = nullptr;
    C_CUDA(cudaSetDevice(device));
    DevBuf buf;
    u32 *ds = nullptr, *dd = nullptr, *dw = nullptr, *row = nullptr, *col = nullptr, *wo = nullptr;
    double *dx = nullptr, *dy = nullptr;
    C_CUDA(buf.alloc(&ds, (size_t)m_in));
    C_CUDA(buf.alloc(&dd, (size_t)m_in));
    C_CUDA(buf.alloc(&dw, (size_t)m_in));
    C_CUDA(buf.alloc(&row, (size_t)n + 1));
    C_CUDA(buf.alloc(&col, (size_t)m_in));
    C_CUDA(buf.alloc(&wo, (size_t)m_in));
    if (x) {
        C_CUDA(buf.alloc(&dx, (size_t)n));
        C_CUDA(buf.alloc(&dy, (size_t)n));
        C_CUDA(cudaMemcpy(dx, x, (size_t)n * 8, cudaMemcpyHostToDevice));
        C_CUDA(cudaMemcpy(dy, y, (size_t)n * 8, cudaMemcpyHostToDevice));
    }
    if (m_in) {
        C_CUDA(cudaMemcpy(ds, src, m_in * 4, cudaMemcpyHostToDevice));
        C_CUDA(cudaMemcpy(dd, dst, m_in * 4, cudaMemcpyHostToDevice));
        C_CUDA(cudaMemcpy(dw, w, m_in * 4, cudaMemcpyHostToDevice));
    }
    pfg_graph_info info;
    pfg_status st = pfg_csr_build_device(n, m_in, ds, dd, dw, dx, dy, row, col, wo, &info, device, nullptr);
    if (st != PFG_OK) return st;
    std::vector<u32> h_row((size_t)n + 1), h_col(info.m), h_w(info.m);
    C_CUDA(cudaMemcpy(h_row.data(), row, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost));
    if (info.m) {
        C_CUDA(cudaMemcpy(h_col.data(), col, (size_t)info.m * 4, cudaMemcpyDeviceToHost));
        C_CUDA(cudaMemcpy(h_w.data(), wo, (size_t)info.m * 4, cudaMemcpyDeviceToHost));
    }
    std::vector<double> hx, hy;
    if (x) {
        hx.assign(x, x + n);
        hy.assign(y, y + n);
    }
    return pfg_internal_graph_from_csr(n, std::move(h_row), std::move(h_col), std::move(h_w), std::move(hx),
                                       std::move(hy), info, out);
}
