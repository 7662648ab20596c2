// mgbvh_exact.cuh — the reference builder's f32 arithmetic, bit for bit.
//
// Every operation here is one IEEE single-precision operation with
// round-to-nearest, in the order the `bvh` crate evaluates it (explicit
// __f*_rn intrinsics, so no FMA contraction and no fast-math division can
// change a bit). The translation unit is also compiled with -fmad=false.
//
//   center .......... bvh/src/lib.rs:71-73   (min + max) * 0.5
//   surface_area .... bvh/src/lib.rs:79-91   2 * ((w*h + w*d) + h*d), 0 if empty
//   is_empty ........ bvh/src/lib.rs:103-106 any(max < min)
//   split cost ...... bvh/src/lib.rs:278-288 (1 + ((SA_lt/SA_p)*8)*n_lt) + ((SA_gt/SA_p)*8)*n_gt
//   bin index ....... bvh/src/lib.rs:358-362 min(floor(((c-cmin)/ext)*bins) as usize, bins-1)
//   threshold ....... bvh/src/lib.rs:430-436 cmin + (ext/steps)*((i as f32) + 0.5)
//   total_cmp ....... f32::total_cmp as an unsigned key (fkey)
//
// Inputs are finite and carry no negative zeros (the builder adds +0.0 to
// every input coordinate), so fminf/fmaxf agree with glam's SSE min/max.
#pragma once

#include <cstdint>

namespace mgbvh {

constexpr float kDepthCost = 1.0f;   // bvh/src/lib.rs:217
constexpr float kObjectCost = 8.0f;  // bvh/src/lib.rs:218

// Order-preserving map float -> u32; the same order as f32::total_cmp.
__host__ __device__ __forceinline__ uint32_t fkey(float f) {
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__host__ __device__ __forceinline__ float funkey(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

constexpr uint32_t kKeyPosInf = 0xFF800000u;  // fkey(+inf): start of a running min
constexpr uint32_t kKeyNegInf = 0x007FFFFFu;  // fkey(-inf): start of a running max

__device__ __forceinline__ float center_of(float lo, float hi) {
    return __fmul_rn(__fadd_rn(lo, hi), 0.5f);
}

__device__ __forceinline__ float surface_area(float lx, float ly, float lz, float hx, float hy,
                                              float hz) {
    if (hx < lx || hy < ly || hz < lz) return 0.0f;
    const float w = __fsub_rn(hx, lx);
    const float h = __fsub_rn(hy, ly);
    const float d = __fsub_rn(hz, lz);
    float s = __fmul_rn(w, h);
    s = __fadd_rn(s, __fmul_rn(w, d));
    s = __fadd_rn(s, __fmul_rn(h, d));
    return __fmul_rn(2.0f, s);
}

__device__ __forceinline__ float surface_area6(const float* b) {
    return surface_area(b[0], b[1], b[2], b[3], b[4], b[5]);
}

__device__ __forceinline__ float split_cost(float sa_lt, float sa_gt, float sa_p, uint32_t n_lt,
                                            uint32_t n_gt) {
    const float lt = __fmul_rn(__fmul_rn(__fdiv_rn(sa_lt, sa_p), kObjectCost), __uint2float_rn(n_lt));
    const float gt = __fmul_rn(__fmul_rn(__fdiv_rn(sa_gt, sa_p), kObjectCost), __uint2float_rn(n_gt));
    return __fadd_rn(__fadd_rn(kDepthCost, lt), gt);
}

__device__ __forceinline__ float leaf_cost(uint32_t len) {  // bvh/src/lib.rs:251-253
    return __fmul_rn(kObjectCost, __uint2float_rn(len));
}

// Bin of centroid coordinate c; ext = cmax - cmin > 0 on this axis.
__device__ __forceinline__ uint32_t bin_of(float c, float cmin, float ext, uint32_t bins) {
    const float pct = __fdiv_rn(__fsub_rn(c, cmin), ext);
    float f = floorf(__fmul_rn(pct, __uint2float_rn(bins)));
    // `as usize` saturates: NaN and negatives map to 0
    f = fminf(f, 4096.0f);
    const uint32_t b = (f > 0.0f) ? static_cast<uint32_t>(f) : 0u;
    return b < bins - 1 ? b : bins - 1;
}

__device__ __forceinline__ float adaptive_threshold(float cmin, float step, uint32_t i) {
    return __fadd_rn(cmin, __fmul_rn(step, __fadd_rn(__uint2float_rn(i), 0.5f)));
}

}  // namespace mgbvh
