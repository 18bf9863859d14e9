// Learned task-cost model: a small MLP (NB_MLP_IN -> 32 -> 32 -> 1, ReLU) with hand-written
// training and inference kernels (sm_100a).  No counterpart in the reference, whose queues
// are ordered by the particle-count-product weights of its METIS partitioner
// (src/engine.c:574-699).
//
// Weights are kept as FP32 master copies and BF16 working copies; forward and backward
// passes read the BF16 copies and accumulate in FP32; Adam updates the master copies and
// re-rounds the working copies.  The network is tiny, so the passes run one sample per
// thread on the FP32 pipe (a tensor-core tile would be >90 % padding).
//
// Parameter layout (NB_MLP_NPARAM floats): W1[32][IN], b1[32], W2[32][32], b2[32], w3[32], b3.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "mdcore_b200.h"

namespace {

constexpr int IN = NB_MLP_IN;
constexpr int H = NB_MLP_HIDDEN;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * IN;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int NP = OFF_B3 + 1;
static_assert(NP == NB_MLP_NPARAM, "parameter count");
constexpr int kThreads = 128;

__device__ __forceinline__ void load_weights(const __nv_bfloat16* __restrict__ w, float* sw) {
    for (int k = threadIdx.x; k < NP; k += blockDim.x) sw[k] = __bfloat162float(w[k]);
    __syncthreads();
}

// Forward pass of one sample; h1, h2 receive the post-ReLU activations.
__device__ __forceinline__ float forward(const float* sw, const float* x, float* h1, float* h2) {
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float a = sw[OFF_B1 + j];
#pragma unroll
        for (int k = 0; k < IN; ++k) a = fmaf(sw[OFF_W1 + j * IN + k], x[k], a);
        h1[j] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float a = sw[OFF_B2 + j];
#pragma unroll
        for (int k = 0; k < H; ++k) a = fmaf(sw[OFF_W2 + j * H + k], h1[k], a);
        h2[j] = fmaxf(a, 0.f);
    }
    float y = sw[OFF_B3];
#pragma unroll
    for (int k = 0; k < H; ++k) y = fmaf(sw[OFF_W3 + k], h2[k], y);
    return y;
}

__global__ void __launch_bounds__(kThreads) mlp_predict_kernel(const float* __restrict__ X, int n,
                                                               const __nv_bfloat16* __restrict__ w,
                                                               float* __restrict__ out) {
    __shared__ float sw[NP];
    load_weights(w, sw);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[IN], h1[H], h2[H];
#pragma unroll
    for (int k = 0; k < IN; ++k) x[k] = X[(size_t)i * IN + k];
    out[i] = forward(sw, x, h1, h2);
}

// Loss = mean over the batch of (y - target)^2; gradients summed into grad (FP32).
__global__ void __launch_bounds__(kThreads) mlp_grad_kernel(const float* __restrict__ X, const float* __restrict__ target,
                                                            const int* __restrict__ idx, int n, float inv_n,
                                                            const __nv_bfloat16* __restrict__ w,
                                                            float* __restrict__ grad, float* __restrict__ loss) {
    __shared__ float sw[NP];
    __shared__ float sg[NP];
    for (int k = threadIdx.x; k < NP; k += blockDim.x) sg[k] = 0.f;
    load_weights(w, sw);
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < n) {
        const int i = idx ? idx[b] : b;
        float x[IN], h1[H], h2[H];
#pragma unroll
        for (int k = 0; k < IN; ++k) x[k] = X[(size_t)i * IN + k];
        const float y = forward(sw, x, h1, h2);
        const float r = y - target[i];
        atomicAdd(loss, r * r * inv_n);
        const float dy = 2.f * r * inv_n;
        atomicAdd(&sg[OFF_B3], dy);
        float dh2[H];
#pragma unroll
        for (int k = 0; k < H; ++k) {
            atomicAdd(&sg[OFF_W3 + k], dy * h2[k]);
            dh2[k] = h2[k] > 0.f ? dy * sw[OFF_W3 + k] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < H; ++j) {
            if (dh2[j] == 0.f) continue;
            atomicAdd(&sg[OFF_B2 + j], dh2[j]);
#pragma unroll
            for (int k = 0; k < H; ++k)
                if (h1[k] > 0.f) atomicAdd(&sg[OFF_W2 + j * H + k], dh2[j] * h1[k]);
        }
#pragma unroll
        for (int k = 0; k < H; ++k) {
            if (h1[k] <= 0.f) continue;
            float d = 0.f;
#pragma unroll
            for (int j = 0; j < H; ++j) d = fmaf(sw[OFF_W2 + j * H + k], dh2[j], d);
            if (d == 0.f) continue;
            atomicAdd(&sg[OFF_B1 + k], d);
#pragma unroll
            for (int m = 0; m < IN; ++m) atomicAdd(&sg[OFF_W1 + k * IN + m], d * x[m]);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NP; k += blockDim.x)
        if (sg[k] != 0.f) atomicAdd(&grad[k], sg[k]);
}

__global__ void mlp_adam_kernel(float* __restrict__ wm, __nv_bfloat16* __restrict__ wb, const float* __restrict__ grad,
                                float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                                float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= NP) return;
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float w = wm[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    wm[k] = w;
    wb[k] = __float2bfloat16_rn(w);
}

__global__ void round_bf16_kernel(const float* __restrict__ wm, __nv_bfloat16* __restrict__ wb, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) wb[k] = __float2bfloat16_rn(wm[k]);
}

}  // namespace

extern "C" int nb_mlp_predict(const float* X, int n, const void* w_bf16, float* out, void* stream) {
    if (n <= 0) return 0;
    mlp_predict_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        X, n, static_cast<const __nv_bfloat16*>(w_bf16), out);
    return cudaGetLastError() == cudaSuccess ? 0 : engine_err_cuda;
}

extern "C" int nb_mlp_grad(const float* X, const float* target, const int* idx, int n, const void* w_bf16,
                           float* grad, float* loss, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(grad, 0, sizeof(float) * NP, s) != cudaSuccess) return engine_err_cuda;
    if (cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) return engine_err_cuda;
    if (n <= 0) return 0;
    mlp_grad_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
        X, target, idx, n, 1.f / (float)n, static_cast<const __nv_bfloat16*>(w_bf16), grad, loss);
    return cudaGetLastError() == cudaSuccess ? 0 : engine_err_cuda;
}

extern "C" int nb_mlp_adam(float* w_master, void* w_bf16, const float* grad, float* m, float* v, float lr,
                           float beta1, float beta2, float eps, int step, void* stream) {
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    mlp_adam_kernel<<<(NP + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w_master, static_cast<__nv_bfloat16*>(w_bf16), grad, m, v, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 0 : engine_err_cuda;
}

extern "C" int nb_mlp_round(const float* w_master, void* w_bf16, void* stream) {
    round_bf16_kernel<<<(NP + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w_master, static_cast<__nv_bfloat16*>(w_bf16), NP);
    return cudaGetLastError() == cudaSuccess ? 0 : engine_err_cuda;
}
