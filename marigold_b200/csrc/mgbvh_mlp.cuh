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

// The builder's copy of the parameters, transposed so that a warp reads one
// input's weights to all 64 units as one 128-byte row (lane l owns units 2l
// and 2l + 1): T1[24][64] b1[64] T2[64][64] b2[64] T3[64][64] b3[64], with
// T[i][j] = W[j][i]; the 49 outputs are padded to 64 with zeros.
constexpr int kTT1 = 0, kTB1 = 1536, kTT2 = 1600, kTB2 = 5696, kTT3 = 5760, kTB3 = 9856;
constexpr int kTParams = 9920;

// Element t of the transposed layout taken from the flat parameter vector.
__host__ __device__ inline int transposed_source(int t) {
    if (t < kTB1) return kOW1 + (t % kH) * kIn + t / kH;
    if (t < kTT2) return kOB1 + (t - kTB1);
    if (t < kTB2) return kOW2 + ((t - kTT2) % kH) * kH + (t - kTT2) / kH;
    if (t < kTT3) return kOB2 + (t - kTB2);
    if (t < kTB3) {
        const int j = (t - kTT3) % kH, i = (t - kTT3) / kH;
        return j < kOut ? kOW3 + j * kH + i : -1;
    }
    const int j = t - kTB3;
    return j < kOut ? kOB3 + j : -1;
}

// One warp evaluates the network on the feature vector `f` (24 floats, the
// same in every lane) with the transposed parameters. Every unit's sum runs
// over its inputs in ascending order, as in the flat-layout passes. Returns,
// in every lane, the best two position outputs (ties to the lower index) and
// the refine logit.
__device__ __forceinline__ void warp_forward_t(const float* f, const __nv_bfloat16* __restrict__ t,
                                               uint32_t lane, int& top0, int& top1,
                                               float& refine) {
    const uint32_t full = 0xFFFFFFFFu;
    const __nv_bfloat162* t2 = reinterpret_cast<const __nv_bfloat162*>(t);
    float h1[2], h2[2];
    {
        const __nv_bfloat162 b = t2[(kTB1 >> 1) + lane];
        float a0 = __low2float(b), a1 = __high2float(b);
#pragma unroll
        for (int i = 0; i < kIn; ++i) {
            const __nv_bfloat162 w = t2[((kTT1 + i * kH) >> 1) + lane];
            a0 += __low2float(w) * f[i];
            a1 += __high2float(w) * f[i];
        }
        h1[0] = gelu(a0);
        h1[1] = gelu(a1);
    }
    {
        const __nv_bfloat162 b = t2[(kTB2 >> 1) + lane];
        float a0 = __low2float(b), a1 = __high2float(b);
#pragma unroll 8
        for (int i = 0; i < kH; ++i) {
            const float x = __shfl_sync(full, (i & 1) ? h1[1] : h1[0], i >> 1);
            const __nv_bfloat162 w = t2[((kTT2 + i * kH) >> 1) + lane];
            a0 += __low2float(w) * x;
            a1 += __high2float(w) * x;
        }
        h2[0] = gelu(a0);
        h2[1] = gelu(a1);
    }
    float o0, o1;
    {
        const __nv_bfloat162 b = t2[(kTB3 >> 1) + lane];
        float a0 = __low2float(b), a1 = __high2float(b);
#pragma unroll 8
        for (int i = 0; i < kH; ++i) {
            const float x = __shfl_sync(full, (i & 1) ? h2[1] : h2[0], i >> 1);
            const __nv_bfloat162 w = t2[((kTT3 + i * kH) >> 1) + lane];
            a0 += __low2float(w) * x;
            a1 += __high2float(w) * x;
        }
        o0 = a0;
        o1 = a1;
    }
    refine = __shfl_sync(full, o0, kPos >> 1);
    // this lane's position outputs: 2 * lane and 2 * lane + 1 (valid below
    // 48); NaN ranks as -inf, and lanes without outputs offer index 0 at -inf,
    // so both results are always valid indices
    const bool ok = 2 * lane < (uint32_t)kPos;
    o0 = (o0 == o0) ? o0 : -INFINITY;
    o1 = (o1 == o1) ? o1 : -INFINITY;
    float bv = ok ? o0 : -INFINITY;
    int bi = ok ? (int)(2 * lane) : 0;
    if (ok && o1 > bv) {
        bv = o1;
        bi = 2 * lane + 1;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(full, bv, off);
        const int oi = __shfl_xor_sync(full, bi, off);
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
        }
    }
    top0 = bi;
    const float c0 = (!ok || (int)(2 * lane) == top0) ? -INFINITY : o0;
    const float c1 = (!ok || (int)(2 * lane + 1) == top0) ? -INFINITY : o1;
    float sv = c0;
    int si = ok ? (int)(2 * lane) : 0;
    if (c1 > sv) {
        sv = c1;
        si = 2 * lane + 1;
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
