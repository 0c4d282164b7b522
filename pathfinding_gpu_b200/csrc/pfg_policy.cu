// pfg_policy.cu - training and batch inference of the learned Delta policy.
//
// The policy is a 12 -> 64 -> 64 -> 64 -> 8 fp32 MLP (ReLU) whose argmax picks
// the next bucket's Delta as a multiple of the automatic Delta (the same
// network is evaluated inside the persistent kernel at every bucket advance,
// see policy_pick in pfg_kernels.cu). It is trained here, on the GPU, with a
// soft-target cross-entropy: each trace row (the features the solver recorded
// at a bucket advance) carries a target distribution over the 8 Delta classes
// derived from the measured run times of fixed-Delta sweeps.
//
// Kernels: k_policy_grad (forward + backward over samples; each CTA of 64
// threads keeps the weights and its gradient slice in shared memory, thread j
// owns neuron j of every hidden layer), k_policy_adam (Adam update), and
// k_policy_infer (one thread per sample). No tensor cores: the network is
// 9.5k parameters and a few thousand samples.
#include "../../include/pfg.h"
#include "pfg_common.cuh"
#include "pfg_internal.h"

#include <cmath>
#include <cstring>
#include <vector>

using namespace pfg;

namespace {

constexpr int NP = (int)(sizeof(PolicyNet) / sizeof(float));
// offsets of the parameter blocks in the flat image
constexpr int O_W1 = 0, O_B1 = O_W1 + POL_H * POL_IN, O_W2 = O_B1 + POL_H, O_B2 = O_W2 + POL_H * POL_H,
              O_W3 = O_B2 + POL_H, O_B3 = O_W3 + POL_H * POL_H, O_W4 = O_B3 + POL_H,
              O_B4 = O_W4 + POL_OUT * POL_H, O_MEAN = O_B4 + POL_OUT, O_SCALE = O_MEAN + POL_IN;
static_assert(O_SCALE + POL_IN == NP, "policy layout");

// Forward + backward of the mean soft-target cross-entropy over `n` samples.
// grad (NP floats, zeroed by the caller) and loss accumulate with atomics.
__global__ void __launch_bounds__(64) k_policy_grad(const float* __restrict__ prm, const float* __restrict__ X,
                                                    const float* __restrict__ Y, u32 n, float* grad, float* loss) {
    extern __shared__ float sm[];
    float* W = sm;              // NP parameters
    float* G = sm + NP;         // NP gradient slots (only weights and biases used)
    float* a0 = G + NP;         // POL_IN
    float* h1 = a0 + POL_IN;    // POL_H each
    float* h2 = h1 + POL_H;
    float* h3 = h2 + POL_H;
    float* z = h3 + POL_H;      // POL_OUT
    float* dz = z + POL_OUT;    // POL_OUT
    float* d3 = dz + POL_OUT;   // POL_H each
    float* d2 = d3 + POL_H;
    float* d1 = d2 + POL_H;
    const int j = threadIdx.x;  // 64 threads
    for (int i = j; i < NP; i += 64) {
        W[i] = prm[i];
        G[i] = 0.f;
    }
    __syncthreads();
    const float inv_n = 1.f / (float)n;
    float my_loss = 0.f;
    for (u32 s = blockIdx.x; s < n; s += gridDim.x) {
        if (j < POL_IN) a0[j] = (X[(size_t)s * POL_IN + j] - W[O_MEAN + j]) * W[O_SCALE + j];
        __syncthreads();
        float acc = W[O_B1 + j];
        for (int i = 0; i < POL_IN; ++i) acc = fmaf(W[O_W1 + j * POL_IN + i], a0[i], acc);
        h1[j] = fmaxf(acc, 0.f);
        __syncthreads();
        acc = W[O_B2 + j];
        for (int i = 0; i < POL_H; ++i) acc = fmaf(W[O_W2 + j * POL_H + i], h1[i], acc);
        h2[j] = fmaxf(acc, 0.f);
        __syncthreads();
        acc = W[O_B3 + j];
        for (int i = 0; i < POL_H; ++i) acc = fmaf(W[O_W3 + j * POL_H + i], h2[i], acc);
        h3[j] = fmaxf(acc, 0.f);
        __syncthreads();
        if (j < POL_OUT) {
            acc = W[O_B4 + j];
            for (int i = 0; i < POL_H; ++i) acc = fmaf(W[O_W4 + j * POL_H + i], h3[i], acc);
            z[j] = acc;
        }
        __syncthreads();
        if (j == 0) {
            // softmax, loss and dL/dz = (p - y) / n
            float mx = z[0];
            for (int o = 1; o < POL_OUT; ++o) mx = fmaxf(mx, z[o]);
            float sum = 0.f;
            for (int o = 0; o < POL_OUT; ++o) sum += expf(z[o] - mx);
            const float lse = mx + logf(sum);
            for (int o = 0; o < POL_OUT; ++o) {
                const float y = Y[(size_t)s * POL_OUT + o];
                const float pr = expf(z[o] - lse);
                my_loss += y * (lse - z[o]);
                dz[o] = (pr - y) * inv_n;
            }
        }
        __syncthreads();
        // layer 4 (thread j owns column j of W4)
        {
            float d = 0.f;
            for (int o = 0; o < POL_OUT; ++o) {
                G[O_W4 + o * POL_H + j] += dz[o] * h3[j];
                d = fmaf(W[O_W4 + o * POL_H + j], dz[o], d);
            }
            if (j < POL_OUT) G[O_B4 + j] += dz[j];
            d3[j] = h3[j] > 0.f ? d : 0.f;
        }
        __syncthreads();
        // layer 3 (thread j owns row j of W3), then dh2[j] = sum_k W3[k][j] d3[k]
        for (int i = 0; i < POL_H; ++i) G[O_W3 + j * POL_H + i] += d3[j] * h2[i];
        G[O_B3 + j] += d3[j];
        {
            float d = 0.f;
            for (int k = 0; k < POL_H; ++k) d = fmaf(W[O_W3 + k * POL_H + j], d3[k], d);
            d2[j] = h2[j] > 0.f ? d : 0.f;
        }
        __syncthreads();
        for (int i = 0; i < POL_H; ++i) G[O_W2 + j * POL_H + i] += d2[j] * h1[i];
        G[O_B2 + j] += d2[j];
        {
            float d = 0.f;
            for (int k = 0; k < POL_H; ++k) d = fmaf(W[O_W2 + k * POL_H + j], d2[k], d);
            d1[j] = h1[j] > 0.f ? d : 0.f;
        }
        __syncthreads();
        for (int i = 0; i < POL_IN; ++i) G[O_W1 + j * POL_IN + i] += d1[j] * a0[i];
        G[O_B1 + j] += d1[j];
        __syncthreads();
    }
    for (int i = j; i < O_MEAN; i += 64)
        if (G[i] != 0.f) atomicAdd(grad + i, G[i]);
    if (j == 0 && my_loss != 0.f) atomicAdd(loss, my_loss * inv_n);
}

// Adam on the trainable part of the image (the input normalisation is fixed).
__global__ void k_policy_adam(float* prm, const float* grad, float* m, float* v, float lr, float b1, float b2,
                              float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O_MEAN) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_policy_infer(const float* __restrict__ prm, const float* __restrict__ X, u32 n, u32* cls) {
    const u32 s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float a0[POL_IN], h1[POL_H], h2[POL_H];
    for (int i = 0; i < POL_IN; ++i) a0[i] = (X[(size_t)s * POL_IN + i] - prm[O_MEAN + i]) * prm[O_SCALE + i];
    for (int j = 0; j < POL_H; ++j) {
        float acc = prm[O_B1 + j];
        for (int i = 0; i < POL_IN; ++i) acc = fmaf(prm[O_W1 + j * POL_IN + i], a0[i], acc);
        h1[j] = fmaxf(acc, 0.f);
    }
    for (int j = 0; j < POL_H; ++j) {
        float acc = prm[O_B2 + j];
        for (int i = 0; i < POL_H; ++i) acc = fmaf(prm[O_W2 + j * POL_H + i], h1[i], acc);
        h2[j] = fmaxf(acc, 0.f);
    }
    for (int j = 0; j < POL_H; ++j) {
        float acc = prm[O_B3 + j];
        for (int i = 0; i < POL_H; ++i) acc = fmaf(prm[O_W3 + j * POL_H + i], h2[i], acc);
        h1[j] = fmaxf(acc, 0.f);  // reuse h1 as layer-3 activations
    }
    int best = 0;
    float bz = -INFINITY;
    for (int o = 0; o < POL_OUT; ++o) {
        float acc = prm[O_B4 + o];
        for (int i = 0; i < POL_H; ++i) acc = fmaf(prm[O_W4 + o * POL_H + i], h1[i], acc);
        if (acc > bz) {
            bz = acc;
            best = o;
        }
    }
    cls[s] = (u32)best;
}

constexpr size_t kGradSmem = (size_t)(2 * NP + POL_IN + 3 * POL_H + 2 * POL_OUT + 3 * POL_H) * sizeof(float);

struct DevBuf {
    std::vector<void*> ptrs;
    ~DevBuf() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T** p, size_t count) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(1, count) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

#define P_CUDA(call)                                                                            \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess) {                                                               \
            cudaGetLastError();                                                                 \
            return set_error(PFG_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e__));    \
        }                                                                                       \
    } while (0)

pfg_status grad_setup() {
    static bool done = false;
    if (!done) {
        P_CUDA(cudaFuncSetAttribute(k_policy_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem));
        done = true;
    }
    return PFG_OK;
}

}  // namespace

extern "C" pfg_status pfg_policy_grad(const float* h_params, const float* h_x, const float* h_y, uint32_t n,
                                      float* h_grad_out, float* loss_out) {
    if (!h_params || !h_x || !h_y || !h_grad_out || n == 0)
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_policy_grad: bad argument");
    pfg_status st = grad_setup();
    if (st != PFG_OK) return st;
    DevBuf b;
    float *dp, *dx, *dy, *dg, *dl;
    P_CUDA(b.alloc(&dp, NP));
    P_CUDA(b.alloc(&dx, (size_t)n * POL_IN));
    P_CUDA(b.alloc(&dy, (size_t)n * POL_OUT));
    P_CUDA(b.alloc(&dg, NP));
    P_CUDA(b.alloc(&dl, 1));
    P_CUDA(cudaMemcpy(dp, h_params, NP * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemcpy(dx, h_x, (size_t)n * POL_IN * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemcpy(dy, h_y, (size_t)n * POL_OUT * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemset(dg, 0, NP * 4));
    P_CUDA(cudaMemset(dl, 0, 4));
    const u32 blocks = std::min<u32>(n, 256u);
    k_policy_grad<<<blocks, 64, kGradSmem>>>(dp, dx, dy, n, dg, dl);
    P_CUDA(cudaGetLastError());
    P_CUDA(cudaMemcpy(h_grad_out, dg, NP * 4, cudaMemcpyDeviceToHost));
    float l = 0.f;
    P_CUDA(cudaMemcpy(&l, dl, 4, cudaMemcpyDeviceToHost));
    for (int i = O_MEAN; i < NP; ++i) h_grad_out[i] = 0.f;
    if (loss_out) *loss_out = l;
    return PFG_OK;
}

extern "C" pfg_status pfg_policy_train(float* h_params, const float* h_x, const float* h_y, uint32_t n,
                                       uint32_t steps, float lr, float* loss_out) {
    if (!h_params || !h_x || !h_y || n == 0 || steps == 0 || !(lr > 0.f))
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_policy_train: bad argument");
    pfg_status st = grad_setup();
    if (st != PFG_OK) return st;
    DevBuf b;
    float *dp, *dx, *dy, *dg, *dl, *dm, *dv;
    P_CUDA(b.alloc(&dp, NP));
    P_CUDA(b.alloc(&dx, (size_t)n * POL_IN));
    P_CUDA(b.alloc(&dy, (size_t)n * POL_OUT));
    P_CUDA(b.alloc(&dg, NP));
    P_CUDA(b.alloc(&dl, steps));
    P_CUDA(b.alloc(&dm, NP));
    P_CUDA(b.alloc(&dv, NP));
    P_CUDA(cudaMemcpy(dp, h_params, NP * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemcpy(dx, h_x, (size_t)n * POL_IN * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemcpy(dy, h_y, (size_t)n * POL_OUT * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemset(dm, 0, NP * 4));
    P_CUDA(cudaMemset(dv, 0, NP * 4));
    P_CUDA(cudaMemset(dl, 0, (size_t)steps * 4));
    const u32 blocks = std::min<u32>(n, 256u);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (u32 t = 1; t <= steps; ++t) {
        P_CUDA(cudaMemsetAsync(dg, 0, NP * 4));
        k_policy_grad<<<blocks, 64, kGradSmem>>>(dp, dx, dy, n, dg, dl + (t - 1));
        const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
        k_policy_adam<<<(O_MEAN + 255) / 256, 256>>>(dp, dg, dm, dv, lr, b1, b2, eps, c1, c2);
    }
    P_CUDA(cudaGetLastError());
    P_CUDA(cudaMemcpy(h_params, dp, NP * 4, cudaMemcpyDeviceToHost));
    if (loss_out) P_CUDA(cudaMemcpy(loss_out, dl, (size_t)steps * 4, cudaMemcpyDeviceToHost));
    return PFG_OK;
}

extern "C" pfg_status pfg_policy_infer(const float* h_params, const float* h_x, uint32_t n, uint32_t* h_class_out) {
    if (!h_params || !h_x || !h_class_out || n == 0)
        return set_error(PFG_ERR_INVALID_ARGUMENT, "pfg_policy_infer: bad argument");
    DevBuf b;
    float *dp, *dx;
    u32* dc;
    P_CUDA(b.alloc(&dp, NP));
    P_CUDA(b.alloc(&dx, (size_t)n * POL_IN));
    P_CUDA(b.alloc(&dc, n));
    P_CUDA(cudaMemcpy(dp, h_params, NP * 4, cudaMemcpyHostToDevice));
    P_CUDA(cudaMemcpy(dx, h_x, (size_t)n * POL_IN * 4, cudaMemcpyHostToDevice));
    k_policy_infer<<<(n + 127) / 128, 128>>>(dp, dx, n, dc);
    P_CUDA(cudaGetLastError());
    P_CUDA(cudaMemcpy(h_class_out, dc, (size_t)n * 4, cudaMemcpyDeviceToHost));
    return PFG_OK;
}
