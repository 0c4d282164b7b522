// pfg_device.cu - device query, warm-up and the host->device transfer study
// (reference: src/gpu_device.cu:39-160), exported through the C ABI.
#include "../../include/pfg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

extern "C" void pfg_internal_set_error(const char* msg);

namespace {
pfg_status dev_fail(pfg_status st, const char* what, cudaError_t e) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    pfg_internal_set_error(buf);
    cudaGetLastError();
    return st;
}
}  // namespace

extern "C" pfg_status pfg_query_device(int32_t dev, pfg_device_info* out) {
    if (!out) return PFG_ERR_INVALID_ARGUMENT;
    memset(out, 0, sizeof(*out));
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= dev || dev < 0) {
        cudaGetLastError();
        return PFG_ERR_NO_DEVICE;
    }
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
        cudaGetLastError();
        return PFG_ERR_CUDA;
    }
    out->ok = 1;
    strncpy(out->name, p.name, sizeof(out->name) - 1);
    out->cc_major = p.major;
    out->cc_minor = p.minor;
    out->sm_count = p.multiProcessorCount;
    out->global_mem = p.totalGlobalMem;
    out->shared_per_block = p.sharedMemPerBlock;
    out->l2_bytes = (uint64_t)p.l2CacheSize;
    out->max_threads_per_sm = p.maxThreadsPerMultiProcessor;
    out->warp_size = p.warpSize;
    int clk = 0, mem_clk = 0, bus = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
    cudaDeviceGetAttribute(&mem_clk, cudaDevAttrMemoryClockRate, dev);
    cudaDeviceGetAttribute(&bus, cudaDevAttrGlobalMemoryBusWidth, dev);
    cudaGetLastError();
    out->clock_mhz = clk / 1000;
    out->mem_clock_mhz = mem_clk / 1000;
    out->bus_width = bus;
    out->peak_bandwidth_gbs = 2.0 * (double)mem_clk * 1e3 * (bus / 8.0) / 1e9;  // double data rate
    cudaDriverGetVersion(&out->driver_version);
    cudaRuntimeGetVersion(&out->runtime_version);
    return PFG_OK;
}

extern "C" pfg_status pfg_warmup(void) {
    cudaError_t e = cudaSetDevice(0);
    if (e == cudaSuccess) e = cudaFree(0);  // creates the context
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? PFG_ERR_NO_DEVICE : PFG_ERR_CUDA;
    }
    return PFG_OK;
}

// Pageable vs pinned vs pinned + 3 streams (8 MB chunks) upload of the CSR.
extern "C" pfg_status pfg_transfer_study_run(const uint32_t* row, const uint32_t* col,
                                             const uint32_t* w, uint32_t n, uint32_t m,
                                             int32_t reps, pfg_transfer_study* out) {
    if (!row || !out || (m && (!col || !w)) || reps <= 0) return PFG_ERR_INVALID_ARGUMENT;
    memset(out, 0, sizeof(*out));
    const size_t bRow = ((size_t)n + 1) * 4, bCol = (size_t)m * 4, bW = (size_t)m * 4;
    out->bytes = (double)(bRow + bCol + bW);
    uint32_t *dRow = nullptr, *dCol = nullptr, *dW = nullptr, *hRow = nullptr, *hCol = nullptr, *hW = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st[3] = {nullptr, nullptr, nullptr};
    pfg_status status = PFG_OK;
    float ms = 0.f;
#define CK(call)                                              \
    do {                                                      \
        cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) {                             \
            status = dev_fail(PFG_ERR_CUDA, #call, e__);      \
            goto done;                                        \
        }                                                     \
    } while (0)
    CK(cudaSetDevice(0));
    CK(cudaMalloc(&dRow, bRow));
    CK(cudaMalloc(&dCol, std::max<size_t>(bCol, 4)));
    CK(cudaMalloc(&dW, std::max<size_t>(bW, 4)));
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int i = 0; i < reps; ++i) {  // (a) pageable
        CK(cudaEventRecord(e0, 0));
        CK(cudaMemcpy(dRow, row, bRow, cudaMemcpyHostToDevice));
        if (m) CK(cudaMemcpy(dCol, col, bCol, cudaMemcpyHostToDevice));
        if (m) CK(cudaMemcpy(dW, w, bW, cudaMemcpyHostToDevice));
        CK(cudaEventRecord(e1, 0));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms, e0, e1));
        out->pageable_ms += ms / reps;
    }
    CK(cudaMallocHost(&hRow, bRow));
    CK(cudaMallocHost(&hCol, std::max<size_t>(bCol, 4)));
    CK(cudaMallocHost(&hW, std::max<size_t>(bW, 4)));
    memcpy(hRow, row, bRow);
    if (m) memcpy(hCol, col, bCol);
    if (m) memcpy(hW, w, bW);
    for (int i = 0; i < reps; ++i) {  // (b) pinned
        CK(cudaEventRecord(e0, 0));
        CK(cudaMemcpyAsync(dRow, hRow, bRow, cudaMemcpyHostToDevice, 0));
        if (m) CK(cudaMemcpyAsync(dCol, hCol, bCol, cudaMemcpyHostToDevice, 0));
        if (m) CK(cudaMemcpyAsync(dW, hW, bW, cudaMemcpyHostToDevice, 0));
        CK(cudaEventRecord(e1, 0));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms, e0, e1));
        out->pinned_ms += ms / reps;
    }
    for (auto& s : st) CK(cudaStreamCreate(&s));
    for (int i = 0; i < reps; ++i) {  // (c) pinned + 3 streams, 8 MB chunks
        CK(cudaEventRecord(e0, 0));
        int sid = 0;
        const size_t CH = 8u << 20;
        const void* srcs[3] = {hRow, hCol, hW};
        void* dsts[3] = {dRow, dCol, dW};
        const size_t sizes[3] = {bRow, bCol, bW};
        for (int a = 0; a < 3; ++a)
            for (size_t off = 0; off < sizes[a]; off += CH) {
                const size_t len = std::min(CH, sizes[a] - off);
                CK(cudaMemcpyAsync((char*)dsts[a] + off, (const char*)srcs[a] + off, len,
                                   cudaMemcpyHostToDevice, st[sid]));
                sid = (sid + 1) % 3;
            }
        for (auto& s : st) CK(cudaStreamSynchronize(s));
        CK(cudaEventRecord(e1, 0));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms, e0, e1));
        out->pinned_streams_ms += ms / reps;
    }
done:
#undef CK
    for (auto& s : st) if (s) cudaStreamDestroy(s);
    if (hRow) cudaFreeHost(hRow);
    if (hCol) cudaFreeHost(hCol);
    if (hW) cudaFreeHost(hW);
    if (dRow) cudaFree(dRow);
    if (dCol) cudaFree(dCol);
    if (dW) cudaFree(dW);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGetLastError();
    return status;
}
