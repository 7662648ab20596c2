// mgbvh_learn.cuh — the learned split proposer inside the builder: node
// features, the exact full-sweep optimum (training labels) and the exact
// scoring of the network's proposals. One warp per node, objects in the
// medium kernel's shared memory (rlo/rhi through an index list).
//
// None of this exists in the reference: the learned form changes the tree
// (by design), while the plain builder stays bit-exact with the reference.
#pragma once

#include <cuda_bf16.h>

#include "mgbvh_device.cuh"
#include "mgbvh_mlp.cuh"

namespace mgbvh {

// Learned-form switches of one build.
struct Learn {
    const __nv_bfloat16* w;  // network parameters; NULL: no proposals
    int gate;                // 1: refine only where the refine logit is > gate_thr
    float* samples;          // training-sample output (kSampleWidth floats each); NULL: none
    uint32_t cap;            // sample capacity
    uint32_t* count;         // samples written (device counter)
    float gate_thr;          // refine-logit threshold of the gate
    uint32_t min_n;          // nodes of fewer objects take the plain split without the network
};

constexpr int kSampleWidth = 30;  // 24 features, label bits, gain, n, plain cost, full cost, start
constexpr uint32_t kSampleLargeMax = 8192;  // level-pass nodes sampled up to this many objects

// Threshold k (0..15) inside proposal bucket `bucket` (0..15) of an axis with
// centroid range [cmin, cmin + ext]: cmin + ext * ((bucket * 16 + k + 1) / 256).
// Nondecreasing in bucket * 16 + k. The fraction is exact: an integer of at
// most 256 times 2^-8 (the same value a division by 256 gives).
__device__ __forceinline__ float proposal_threshold(float cmin, float ext, uint32_t bucket, uint32_t k) {
    return __fadd_rn(cmin, __fmul_rn(ext, __fmul_rn((float)(bucket * 16u + k + 1u), 0.00390625f)));
}

// A level-pass node waiting for its proposals to be scored.
struct LvlRefine {
    uint32_t on;       // 1: proposals pending (the node's split is decided after the refine pass)
    uint32_t prop[2];  // axis * 16 + bucket
    uint32_t pad;
};
// interval bins of a pending level-pass node: [proposal][interval 0..16]{count, lo key xyz, hi key xyz};
// interval j holds the centroids c with thr[j - 1] <= c < thr[j]
constexpr uint32_t kRBinWords = 2 * 17 * 7;

// One training sample (lane 0 of the calling warp): features f, the
// full-sweep optimum (cost key bk, axis ba, threshold bthr; bk == kNoKey:
// none), the centroid range of axis ba, the binned split's cost key, the
// object count and the node's start in its object list.
__device__ __forceinline__ void write_sample(const Learn& LN, const float* f, uint32_t bk, uint32_t ba,
                                             float bthr, float cmin_a, float ext_a, uint32_t plain_ck,
                                             uint32_t n, uint32_t start) {
    const uint32_t slot = atomicAdd(LN.count, 1u);
    if (slot >= LN.cap) return;
    float* out = LN.samples + (size_t)slot * kSampleWidth;
    for (int j = 0; j < 24; ++j) out[j] = f[j];
    uint32_t label = 0xFFFFFFFFu;
    float gain = 0.0f;
    if (bk != kNoKey && ext_a > 0.0f) {
        const float pct = (bthr - cmin_a) / ext_a;
        int q = (int)floorf(pct * 16.0f);
        q = min(max(q, 0), 15);
        label = ba * 16u + (uint32_t)q;
        gain = bk < plain_ck ? 1.0f : 0.0f;
    }
    out[24] = __uint_as_float(label);
    out[25] = gain;
    out[26] = (float)n;
    out[27] = funkey(plain_ck);
    out[28] = bk == kNoKey ? __int_as_float(0x7F800000) : funkey(bk);
    out[29] = (float)start;
}

// Node features (every lane gets all 24). nb: node bounds; cb: centroid
// bounds (lo xyz, hi xyz); cnt: this lane's 32-bin counts per axis (lane =
// bin), so the 4-bucket histogram of an axis is the sum of 8 adjacent bins.
__device__ __forceinline__ void node_features(const float* nb, const float* cb, uint32_t n,
                                              uint32_t depth, const uint32_t* cnt, float* f) {
    float ext[3], cext[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ext[a] = nb[3 + a] - nb[a];
        cext[a] = cb[3 + a] - cb[a];
    }
    const float emax = fmaxf(fmaxf(ext[0], ext[1]), fmaxf(ext[2], 1e-30f));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        f[a] = ext[a] / emax;
        f[3 + a] = cext[a] / emax;
    }
    f[6] = log2f((float)n) / 20.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        uint32_t c = cnt[a];
        // sum over the 8 lanes of each group of 8 bins
        c += __shfl_xor_sync(kFull, c, 1);
        c += __shfl_xor_sync(kFull, c, 2);
        c += __shfl_xor_sync(kFull, c, 4);
#pragma unroll
        for (int q = 0; q < 4; ++q) f[7 + 4 * a + q] = (float)__shfl_sync(kFull, c, 8 * q) / (float)n;
    }
    const float sap = surface_area6(nb);
    f[19] = sap > 0.0f ? surface_area6(cb) / sap : 0.0f;
    f[20] = (float)depth / 32.0f;
    float lo = fminf(fminf(ext[0], ext[1]), ext[2]);
    float hi = fmaxf(fmaxf(ext[0], ext[1]), ext[2]);
    float mid = ext[0] + ext[1] + ext[2] - lo - hi;
    // exact middle: the one that is neither the min nor the max position
    {
        int imin = 0, imax = 0;
        for (int a = 1; a < 3; ++a) {
            if (ext[a] < ext[imin]) imin = a;
            if (ext[a] > ext[imax] || (ext[a] == ext[imax] && imax == imin)) imax = a;
        }
        if (imin == imax) imax = (imin + 1) % 3;
        mid = ext[3 - imin - imax];
    }
    f[21] = mid / emax;
    f[22] = lo / emax;
    f[23] = fmaxf(fmaxf(cext[0], cext[1]), cext[2]) / emax;
    (void)hi;
}

// Threshold split scoring over the node's objects for one threshold per
// lane: returns this lane's candidate (cost key etc.) in `c`.
template <class Fetch>
__device__ __forceinline__ void score_threshold(Fetch fetch, uint32_t n, uint32_t axis, float thr,
                                                bool active, float sa_p, const Params& P, Cand& c,
                                                uint32_t idx) {
    float blt[6], bgt[6];
    box_empty(blt);
    box_empty(bgt);
    uint32_t nl = 0;
    for (uint32_t j = 0; j < n; ++j) {
        float lo[3], hi[3];
        fetch(j, lo, hi);
        const float cj = center_of(axis == 0 ? lo[0] : (axis == 1 ? lo[1] : lo[2]),
                                   axis == 0 ? hi[0] : (axis == 1 ? hi[1] : hi[2]));
        if (cj < thr) {
            box_grow(blt, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
            nl++;
        } else {
            box_grow(bgt, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
        }
    }
    c.key = ~0ull;
    const uint32_t ng = n - nl;
    if (active && nl >= P.min_leaf && ng >= P.min_leaf) {
        const float cost = split_cost(surface_area6(blt), surface_area6(bgt), sa_p, nl, ng);
        c.key = cand_key(cost, axis, idx);
        c.n_lt = nl;
        c.thr = thr;
        for (int i = 0; i < 6; ++i) {
            c.lt[i] = blt[i];
            c.gt[i] = bgt[i];
        }
    }
}

}  // namespace mgbvh
