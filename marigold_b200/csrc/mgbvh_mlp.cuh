// mgbvh_mlp.cuh — the learned split proposer's network: layout, activation
// and the one-warp forward pass used inside the builder.
//
// 24 -> 64 -> 64 -> 49, exact GELU, BF16 parameters, FP32 accumulation.
// Flat parameter vector: W1[64x24] b1[64] W2[64x64] b2[64] W3[49x64] b3[49].
// Outputs 0..47: split-position logits (axis * 16 + bucket, 16 equal buckets
// over the node's centroid extent on that axis); output 48: refine logit (the
// exact evaluation near the proposals is worth running).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace mgbvh_mlp {

constexpr int kIn = 24, kH = 64, kOut = 49, kPos = 48;
constexpr int kOW1 = 0, kOB1 = 1536, kOW2 = 1600, kOB2 = 5696, kOW3 = 5760, kOB3 = 8896;
constexpr int kParams = 8945;
constexpr uint32_t kNoLabel = 0xFFFFFFFFu;

__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ float wv(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// One warp evaluates the network on one feature vector held in `f` (24
// floats, the same in every lane). Returns, in every lane, the best two
// position outputs (index, logit) and the refine logit.
__device__ __forceinline__ void warp_forward(const float* f, const __nv_bfloat16* __restrict__ w,
                                             uint32_t lane, int& top0, int& top1,
                                             float& refine) {
    const uint32_t full = 0xFFFFFFFFu;
    float h1[2], h2[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int j = lane + 32 * r;
        float acc = wv(w, kOB1 + j);
#pragma unroll
        for (int i = 0; i < kIn; ++i) acc += wv(w, kOW1 + j * kIn + i) * f[i];
        h1[r] = gelu(acc);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int j = lane + 32 * r;
        float acc = wv(w, kOB2 + j);
        for (int i = 0; i < kH; ++i) {
            const float a = __shfl_sync(full, h1[i >> 5], i & 31);
            acc += wv(w, kOW2 + j * kH + i) * a;
        }
        h2[r] = gelu(acc);
    }
    float o[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int j = lane + 32 * r;
        float acc = j < kOut ? wv(w, kOB3 + j) : 0.0f;
        for (int i = 0; i < kH; ++i) {
            const float a = __shfl_sync(full, h2[i >> 5], i & 31);
            if (j < kOut) acc += wv(w, kOW3 + j * kH + i) * a;
        }
        o[r] = acc;
    }
    refine = __shfl_sync(full, o[1], kPos - 32);
    // top two of the 48 position logits (ties to the lower index)
    float v0 = o[0];
    int i0 = lane;
    const float v1 = lane + 32 < kPos ? o[1] : -INFINITY;
    if (v1 > v0) {
        v0 = v1;
        i0 = lane + 32;
    }
    float bv = v0;
    int bi = i0;
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(full, bv, off);
        const int oi = __shfl_xor_sync(full, bi, off);
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
        }
    }
    top0 = bi;
    // second best: the best of the rest
    float c0 = (lane == (uint32_t)top0) ? -INFINITY : o[0];
    float c1 = (lane + 32 == (uint32_t)top0 || lane + 32 >= (uint32_t)kPos) ? -INFINITY : o[1];
    float sv = c0;
    int si = lane;
    if (c1 > sv) {
        sv = c1;
        si = lane + 32;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(full, sv, off);
        const int oi = __shfl_xor_sync(full, si, off);
        if (ov > sv || (ov == sv && oi < si)) {
            sv = ov;
            si = oi;
        }
    }
    top1 = si;
}

}  // namespace mgbvh_mlp
