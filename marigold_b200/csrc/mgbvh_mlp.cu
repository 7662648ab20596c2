// mgbvh_mlp.cu — training and batch inference of the learned split proposer.
//
// The network (layout in mgbvh_mlp.cuh) is trained on node samples whose
// label is the exact full-sweep SAH optimum (axis and position bucket) and
// whether it beats the plain binned split. Parameters are BF16 in the
// forward and backward passes, with FP32 accumulation; the optimizer keeps
// FP32 master weights (Adam) and rewrites the BF16 copy after each step.
//
// One CTA handles 32 samples: weights (as FP32) and activations in shared
// memory, forward through both hidden layers, softmax cross-entropy over the
// 48 position logits plus binary cross-entropy of the refine logit, then the
// backward pass; each CTA adds its parameter gradients to the global FP32
// gradient with one atomic per parameter.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mgbvh.h"
#include "mgbvh_mlp.cuh"

namespace mgbvh_mlp {

constexpr int kSB = 32;  // samples per CTA
constexpr int kThreads = 256;

struct TrainSmem {
    float w[kParams];
    float x[kSB][kIn];
    float z1[kSB][kH], a1[kSB][kH];
    float z2[kSB][kH], a2[kSB][kH];
    float d3[kSB][kOut];
    float d2[kSB][kH];
    float d1[kSB][kH];
    float loss[2];
};

__device__ void forward_block(TrainSmem& S, int ns) {
    const int tid = threadIdx.x;
    for (int idx = tid; idx < kSB * kH; idx += kThreads) {
        const int s = idx / kH, j = idx % kH;
        float acc = S.w[kOB1 + j];
        for (int i = 0; i < kIn; ++i) acc += S.w[kOW1 + j * kIn + i] * S.x[s][i];
        S.z1[s][j] = acc;
        S.a1[s][j] = gelu(acc);
    }
    __syncthreads();
    for (int idx = tid; idx < kSB * kH; idx += kThreads) {
        const int s = idx / kH, j = idx % kH;
        float acc = S.w[kOB2 + j];
        for (int i = 0; i < kH; ++i) acc += S.w[kOW2 + j * kH + i] * S.a1[s][i];
        S.z2[s][j] = acc;
        S.a2[s][j] = gelu(acc);
    }
    __syncthreads();
    for (int idx = tid; idx < kSB * kOut; idx += kThreads) {
        const int s = idx / kOut, o = idx % kOut;
        float acc = S.w[kOB3 + o];
        for (int i = 0; i < kH; ++i) acc += S.w[kOW3 + o * kH + i] * S.a2[s][i];
        S.d3[s][o] = acc;  // logits; turned into gradients below
    }
    __syncthreads();
    (void)ns;
}

__device__ void load_block(TrainSmem& S, const float* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                           uint32_t base, int ns) {
    const int tid = threadIdx.x;
    for (int i = tid; i < kParams; i += kThreads) S.w[i] = __bfloat162float(w[i]);
    for (int i = tid; i < kSB * kIn; i += kThreads) {
        const int s = i / kIn;
        S.x[s][i % kIn] = s < ns ? x[(size_t)(base + s) * kIn + (i % kIn)] : 0.0f;
    }
    if (tid < 2) S.loss[tid] = 0.0f;
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) train_kernel(const float* __restrict__ x,
                                                        const uint32_t* __restrict__ label,
                                                        const float* __restrict__ gain, uint32_t B,
                                                        const __nv_bfloat16* __restrict__ w,
                                                        float* __restrict__ grad, float* loss) {
    extern __shared__ __align__(16) unsigned char raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(raw);
    const uint32_t base = blockIdx.x * kSB;
    const int ns = (int)min((uint32_t)kSB, B - base);
    const int tid = threadIdx.x;
    load_block(S, x, w, base, ns);
    forward_block(S, ns);
    // output gradients (mean over the batch: scale 1/B)
    const float invB = 1.0f / (float)B;
    if (tid < kSB) {
        const int s = tid;
        if (s < ns) {
            const uint32_t lab = label[base + s];
            const float g = gain[base + s];
            float ce = 0.0f;
            if (lab < (uint32_t)kPos) {  // kNoLabel and anything out of range: no position loss
                float m = -INFINITY;
                for (int o = 0; o < kPos; ++o) m = fmaxf(m, S.d3[s][o]);
                float sum = 0.0f;
                for (int o = 0; o < kPos; ++o) sum += expf(S.d3[s][o] - m);
                ce = logf(sum) + m - S.d3[s][lab];
                for (int o = 0; o < kPos; ++o)
                    S.d3[s][o] = (expf(S.d3[s][o] - m) / sum - (o == (int)lab ? 1.0f : 0.0f)) * invB;
            } else {
                for (int o = 0; o < kPos; ++o) S.d3[s][o] = 0.0f;
            }
            const float l = S.d3[s][kPos];
            const float sig = 1.0f / (1.0f + expf(-l));
            const float bce = fmaxf(l, 0.0f) + log1pf(expf(-fabsf(l))) - g * l;
            S.d3[s][kPos] = (sig - g) * invB;
            atomicAdd(&S.loss[0], ce);
            atomicAdd(&S.loss[1], bce);
        } else {
            for (int o = 0; o < kOut; ++o) S.d3[s][o] = 0.0f;
        }
    }
    __syncthreads();
    if (tid == 0) {
        atomicAdd(&loss[0], S.loss[0]);
        atomicAdd(&loss[1], S.loss[1]);
    }
    // W3, b3 gradients; d2 = (d3 W3) * gelu'(z2)
    for (int idx = tid; idx < kOut * kH + kOut; idx += kThreads) {
        float acc = 0.0f;
        if (idx < kOut * kH) {
            const int o = idx / kH, j = idx % kH;
            for (int s = 0; s < kSB; ++s) acc += S.d3[s][o] * S.a2[s][j];
            atomicAdd(&grad[kOW3 + idx], acc);
        } else {
            const int o = idx - kOut * kH;
            for (int s = 0; s < kSB; ++s) acc += S.d3[s][o];
            atomicAdd(&grad[kOB3 + o], acc);
        }
    }
    for (int idx = tid; idx < kSB * kH; idx += kThreads) {
        const int s = idx / kH, j = idx % kH;
        float acc = 0.0f;
        for (int o = 0; o < kOut; ++o) acc += S.w[kOW3 + o * kH + j] * S.d3[s][o];
        S.d2[s][j] = acc * gelu_grad(S.z2[s][j]);
    }
    __syncthreads();
    for (int idx = tid; idx < kH * kH + kH; idx += kThreads) {
        float acc = 0.0f;
        if (idx < kH * kH) {
            const int j = idx / kH, i = idx % kH;
            for (int s = 0; s < kSB; ++s) acc += S.d2[s][j] * S.a1[s][i];
            atomicAdd(&grad[kOW2 + idx], acc);
        } else {
            const int j = idx - kH * kH;
            for (int s = 0; s < kSB; ++s) acc += S.d2[s][j];
            atomicAdd(&grad[kOB2 + j], acc);
        }
    }
    for (int idx = tid; idx < kSB * kH; idx += kThreads) {
        const int s = idx / kH, i = idx % kH;
        float acc = 0.0f;
        for (int j = 0; j < kH; ++j) acc += S.w[kOW2 + j * kH + i] * S.d2[s][j];
        S.d1[s][i] = acc * gelu_grad(S.z1[s][i]);
    }
    __syncthreads();
    for (int idx = tid; idx < kH * kIn + kH; idx += kThreads) {
        float acc = 0.0f;
        if (idx < kH * kIn) {
            const int j = idx / kIn, i = idx % kIn;
            for (int s = 0; s < kSB; ++s) acc += S.d1[s][j] * S.x[s][i];
            atomicAdd(&grad[kOW1 + idx], acc);
        } else {
            const int j = idx - kH * kIn;
            for (int s = 0; s < kSB; ++s) acc += S.d1[s][j];
            atomicAdd(&grad[kOB1 + j], acc);
        }
    }
}

__global__ void __launch_bounds__(kThreads) forward_kernel(const float* __restrict__ x, uint32_t B,
                                                          const __nv_bfloat16* __restrict__ w,
                                                          float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(raw);
    const uint32_t base = blockIdx.x * kSB;
    const int ns = (int)min((uint32_t)kSB, B - base);
    load_block(S, x, w, base, ns);
    forward_block(S, ns);
    for (int idx = threadIdx.x; idx < ns * kOut; idx += kThreads)
        out[(size_t)(base + idx / kOut) * kOut + idx % kOut] = S.d3[idx / kOut][idx % kOut];
}

// Adam on FP32 master weights; writes the BF16 copy used by the passes.
__global__ void adam_kernel(float* __restrict__ master, __nv_bfloat16* __restrict__ w,
                            const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    master[i] = p;
    w[i] = __float2bfloat16_rn(p);
}

}  // namespace mgbvh_mlp

using namespace mgbvh_mlp;

extern "C" {

int mgbvh_mlp_train_step_dev(const float* d_features, const uint32_t* d_labels, const float* d_gains,
                             uint32_t batch, const void* d_weights_bf16, float* d_grad,
                             float* d_loss, void* stream) {
    if (!d_features || !d_labels || !d_gains || !d_weights_bf16 || !d_grad || !d_loss || batch == 0)
        return MGBVH_ERR_INVALID_ARG;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(TrainSmem)) != cudaSuccess ||
            cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(TrainSmem)) != cudaSuccess)
            return MGBVH_ERR_CUDA;
        attr = true;
    }
    train_kernel<<<(batch + kSB - 1) / kSB, kThreads, sizeof(TrainSmem),
                   reinterpret_cast<cudaStream_t>(stream)>>>(
        d_features, d_labels, d_gains, batch, static_cast<const __nv_bfloat16*>(d_weights_bf16), d_grad,
        d_loss);
    return cudaGetLastError() == cudaSuccess ? MGBVH_OK : MGBVH_ERR_CUDA;
}

int mgbvh_mlp_forward_dev(const float* d_features, uint32_t batch, const void* d_weights_bf16,
                          float* d_out, void* stream) {
    if (!d_features || !d_weights_bf16 || !d_out) return MGBVH_ERR_INVALID_ARG;
    if (batch == 0) return MGBVH_OK;
    if (cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(TrainSmem)) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    forward_kernel<<<(batch + kSB - 1) / kSB, kThreads, sizeof(TrainSmem),
                     reinterpret_cast<cudaStream_t>(stream)>>>(
        d_features, batch, static_cast<const __nv_bfloat16*>(d_weights_bf16), d_out);
    return cudaGetLastError() == cudaSuccess ? MGBVH_OK : MGBVH_ERR_CUDA;
}

int mgbvh_mlp_adam_dev(float* d_master, void* d_weights_bf16, const float* d_grad, float* d_m,
                       float* d_v, uint32_t step, float lr, float beta1, float beta2, float eps,
                       void* stream) {
    if (!d_master || !d_weights_bf16 || !d_grad || !d_m || !d_v || step == 0) return MGBVH_ERR_INVALID_ARG;
    const float bc1 = 1.0f - powf(beta1, (float)step);
    const float bc2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<(kParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        d_master, static_cast<__nv_bfloat16*>(d_weights_bf16), d_grad, d_m, d_v, lr, beta1, beta2, eps,
        bc1, bc2);
    return cudaGetLastError() == cudaSuccess ? MGBVH_OK : MGBVH_ERR_CUDA;
}

}  // extern "C"
