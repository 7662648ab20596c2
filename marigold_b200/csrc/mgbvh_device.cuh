// mgbvh_device.cuh — device-side types and the warp subtree builder.
//
// A subtree whose root holds at most 32 objects is built by one warp with
// the objects in registers: lane i holds the object at position i of the
// subtree's range. The warp visits the subtree's nodes depth first; for each
// node it evaluates every candidate split of the reference's select_split
// (bvh/src/lib.rs:493-534) in parallel, one candidate per lane, and applies
// the winner with a stable ballot partition of the lanes.
#pragma once

#include <cstdint>

#include "mgbvh_exact.cuh"
#include "../../include/mgbvh.h"

namespace mgbvh {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kSmallMax = 32;  // warp subtree size
constexpr uint32_t kMaxBins = 32;
constexpr uint32_t kNoKey = 0xFFFFFFFFu;

// Split parameters, the const generics and BvhSettings of the crate.
struct Params {
    uint32_t min_leaf;        // MIN_LEAF_OBJECTS
    uint32_t max_leaf;        // MAX_LEAF_OBJECTS
    uint32_t max_depth;       // BvhSettings::max_depth
    uint32_t bins;            // 0: len.clamp(16,32)
    uint32_t adaptive_max_n;  // adaptive sweep for len <= this (<= 32)
    uint32_t adaptive_steps;  // 0: len.clamp(8,32)
    uint32_t medium_max;      // nodes above this go through the level passes (<= 1024)
};

// Streamed output: the node slots split into kStreamChunks ranges; a subtree
// of <= 32 objects whose children pair starts in range c is built by the
// c-th launch of the small kernel.
constexpr uint32_t kStreamChunks = 8;

__host__ __device__ __forceinline__ uint32_t stream_chunk(uint32_t pair, uint32_t slots) {
    const uint32_t c = static_cast<uint32_t>((static_cast<uint64_t>(pair) * kStreamChunks) / slots);
    return c < kStreamChunks ? c : kStreamChunks - 1u;
}

// First slot of chunk c (c = kStreamChunks: the slot count).
__host__ __device__ __forceinline__ uint32_t stream_chunk_begin(uint32_t c, uint32_t slots) {
    return static_cast<uint32_t>((static_cast<uint64_t>(c) * slots + kStreamChunks - 1u) / kStreamChunks);
}

// Device counters and flags of one build.
struct Counters {
    uint32_t error;         // first mgbvh_status error code, 0 if none
    uint32_t error_site;    // which check failed (for messages)
    uint32_t height;        // max depth of a split node (bvh/src/lib.rs:656)
    uint32_t median_splits;
    uint32_t depth_capped;  // leaves cut by max_depth holding > 1 object
    uint32_t holes;         // leaves holding > 1 object (node slots to compact)
    uint32_t lvl[3][2];     // [level % 3] {large tasks, tiles} of a level pass
    uint32_t n_medium;
    uint32_t n_small;
    uint32_t root_keys[12];  // object bounds lo/hi keys, centroid lo/hi keys
    uint32_t learned;        // nodes where a proposal of the split network replaced the binned split
    uint32_t n_med;          // level-pass nodes waiting for a forced median split (the median passes)
    uint32_t medium_take;    // next subtree CTA task to take (subtree CTAs take tasks in turn)
    uint32_t small_take;     // next small-subtree task to take (warps take tasks in turn)
    uint32_t mtake[8];       // streamed output: the same, per slot chunk (subtree CTA tasks)
    uint32_t stake[8];       // streamed output: the same, per slot chunk (small-subtree tasks)
    // streamed output (slot chunks): subtrees of 33..medium_max objects per
    // chunk, their placement cursors and sorted ranges; subtrees of <= 32
    // objects selected so far, the sorted range of each chunk's, and the CTAs
    // of each chunk's selection pass that finished
    uint32_t mbk[8];
    uint32_t mbcur[8];
    uint32_t mrange[9];
    uint32_t s2n;
    uint32_t srange[9];
    uint32_t sdone[8];
};

enum ErrorSite : uint32_t {
    kSiteNone = 0,
    kSiteIndex = 1,        // a triangle index past the vertex count
    kSiteCount = 2,        // partition count differs from the split's count
    kSiteContain = 3,      // a centroid outside its child's bounds
    kSiteMedian = 4,       // forced median of a level-pass node: counts of its halves differ
    kSiteCapacity = 5,
    kSiteMeshIndex = 6,  // an instance names a mesh past the mesh count
};

__device__ __forceinline__ void set_error(Counters* c, int status, uint32_t site) {
    if (atomicCAS(&c->error, 0u, static_cast<uint32_t>(status)) == 0u) c->error_site = site;
}

// Where a finished node goes. Node slots follow the reference's numbering
// (pre-order over child pairs, gt child first, bvh/src/lib.rs:650-663),
// computed in closed form under the assumption that every leaf holds one
// object: the gt child of a node whose children sit at P has its children at
// P + 2, the lt child at P + 2 * len_gt. Leaves with more objects leave
// unused slots ("holes") that a compaction pass removes afterwards.
struct Out {
    mgbvh_node* nodes;
    uint32_t* lens;
    uint8_t* used;
    uint32_t* perm;
    Counters* ctr;
    uint32_t node_cap;  // slots in nodes/lens/used
};

// The 8 words of a node are written by lanes 0..7 (one 32-byte store), the
// length by lane 8 and the used flag by lane 9. All arguments warp-uniform.
__device__ __forceinline__ void warp_store_node(const Out& o, uint32_t slot, const float* b,
                                                uint32_t start, uint32_t len, uint32_t child,
                                                uint32_t lane) {
    if (slot >= o.node_cap) {  // cannot happen with the closed-form slots; never write past
        if (lane == 0) set_error(o.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
        return;
    }
    uint32_t w = 0;
    switch (lane) {
        case 0: w = __float_as_uint(b[0]); break;
        case 1: w = __float_as_uint(b[1]); break;
        case 2: w = __float_as_uint(b[2]); break;
        case 3: w = start; break;
        case 4: w = __float_as_uint(b[3]); break;
        case 5: w = __float_as_uint(b[4]); break;
        case 6: w = __float_as_uint(b[5]); break;
        case 7: w = child; break;
        default: break;
    }
    if (lane < 8) reinterpret_cast<uint32_t*>(o.nodes + slot)[lane] = w;
    if (lane == 8) o.lens[slot] = len;
    if (lane == 9) o.used[slot] = 1;
}

__device__ __forceinline__ void box_empty(float* b) {
    b[0] = b[1] = b[2] = __int_as_float(0x7F800000);
    b[3] = b[4] = b[5] = __int_as_float(0xFF800000);
}

__device__ __forceinline__ void box_grow(float* b, float lx, float ly, float lz, float hx, float hy,
                                         float hz) {
    b[0] = fminf(b[0], lx);
    b[1] = fminf(b[1], ly);
    b[2] = fminf(b[2], lz);
    b[3] = fmaxf(b[3], hx);
    b[4] = fmaxf(b[4], hy);
    b[5] = fmaxf(b[5], hz);
}

__device__ __forceinline__ bool box_contains(const float* b, float x, float y, float z) {
    const bool empty = b[3] < b[0] || b[4] < b[1] || b[5] < b[2];
    return !empty && x >= b[0] && y >= b[1] && z >= b[2] && x <= b[3] && y <= b[4] && z <= b[5];
}

// v[i] for i < 3 with selects: a run-time index into a local array would
// put the array in local memory.
__device__ __forceinline__ float sel3(const float* v, uint32_t i) {
    return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]);
}

// box_contains on box a (first) or box b, chosen with selects on constant
// indexes (a pointer chosen at run time would put both boxes in local memory).
__device__ __forceinline__ bool box_contains2(const float* a, const float* b, bool first, float x, float y,
                                              float z) {
    float bb[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) bb[i] = first ? a[i] : b[i];
    return box_contains(bb, x, y, z);
}

// box_grow on box a (first) or box b, with selects on constant indexes.
__device__ __forceinline__ void box_grow2(float* a, float* b, bool first, float lx, float ly, float lz,
                                          float hx, float hy, float hz) {
    const float l[3] = {lx, ly, lz}, h[3] = {hx, hy, hz};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        a[i] = first ? fminf(a[i], l[i]) : a[i];
        a[3 + i] = first ? fmaxf(a[3 + i], h[i]) : a[3 + i];
        b[i] = first ? b[i] : fminf(b[i], l[i]);
        b[3 + i] = first ? b[3 + i] : fmaxf(b[3 + i], h[i]);
    }
}

// Warp union of the boxes of the lanes in `mask` (exact: min/max on keys).
__device__ __forceinline__ void warp_box_union(bool in, const float* lo, const float* hi,
                                               float* out) {
    for (int a = 0; a < 3; ++a) {
        out[a] = funkey(__reduce_min_sync(kFull, in ? fkey(lo[a]) : kKeyPosInf));
        out[3 + a] = funkey(__reduce_max_sync(kFull, in ? fkey(hi[a]) : kKeyNegInf));
    }
}

// 64-bit candidate key: total_cmp(cost), then axis, then candidate index —
// the first minimum of min_by over axes of min_by over candidates.
__device__ __forceinline__ uint64_t cand_key(float cost, uint32_t axis, uint32_t idx) {
    return (static_cast<uint64_t>(fkey(cost)) << 32) | (axis << 8) | idx;
}

// Warp-wide minimum of 64-bit keys via two 32-bit reductions.
__device__ __forceinline__ uint64_t warp_min_key(uint64_t k) {
    const uint32_t hi = static_cast<uint32_t>(k >> 32), lo = static_cast<uint32_t>(k);
    const uint32_t mh = __reduce_min_sync(kFull, hi);
    const uint32_t ml = __reduce_min_sync(kFull, hi == mh ? lo : kNoKey);
    return (static_cast<uint64_t>(mh) << 32) | ml;
}

// Prefix (inclusive) and suffix (inclusive) unions across lanes of one
// axis's bins: count and box. Lanes at or past `bins` carry empty bins.
struct BinScan {
    uint32_t pre_cnt, suf_cnt;
    float pre[6], suf[6];
};

__device__ __forceinline__ void bin_scan(uint32_t cnt, const float* box, uint32_t lane,
                                         BinScan& s) {
    s.pre_cnt = cnt;
    s.suf_cnt = cnt;
    for (int i = 0; i < 6; ++i) s.pre[i] = s.suf[i] = box[i];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t pc = __shfl_up_sync(kFull, s.pre_cnt, off);
        const uint32_t sc = __shfl_down_sync(kFull, s.suf_cnt, off);
        float pv[6], sv[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            pv[i] = __shfl_up_sync(kFull, s.pre[i], off);
            sv[i] = __shfl_down_sync(kFull, s.suf[i], off);
        }
        if (lane >= static_cast<uint32_t>(off)) {
            s.pre_cnt += pc;
            s.pre[0] = fminf(s.pre[0], pv[0]);
            s.pre[1] = fminf(s.pre[1], pv[1]);
            s.pre[2] = fminf(s.pre[2], pv[2]);
            s.pre[3] = fmaxf(s.pre[3], pv[3]);
            s.pre[4] = fmaxf(s.pre[4], pv[4]);
            s.pre[5] = fmaxf(s.pre[5], pv[5]);
        }
        if (lane + off < 32u) {
            s.suf_cnt += sc;
            s.suf[0] = fminf(s.suf[0], sv[0]);
            s.suf[1] = fminf(s.suf[1], sv[1]);
            s.suf[2] = fminf(s.suf[2], sv[2]);
            s.suf[3] = fmaxf(s.suf[3], sv[3]);
            s.suf[4] = fmaxf(s.suf[4], sv[4]);
            s.suf[5] = fmaxf(s.suf[5], sv[5]);
        }
    }
}

// Best binned candidate held by this lane over the three axes
// (evaluate_binned_split for split index i = lane, bvh/src/lib.rs:255-290,
// 373-388). cnt/box: this lane's bin (lane = bin index) per axis.
struct Cand {
    uint64_t key;
    uint32_t n_lt;
    float lt[6], gt[6];
    float thr;  // adaptive threshold (unused for binned)
};

// load(a, cnt, box6): this lane's bin on axis a.
template <class Load>
__device__ __forceinline__ void binned_candidates_f(Load load, const bool* axis_ok, uint32_t bins,
                                                    uint32_t n, float sa_p, const Params& P,
                                                    uint32_t lane, Cand& best) {
    best.key = ~0ull;
#pragma unroll 1
    for (uint32_t a = 0; a < 3; ++a) {
        // selects, not a run-time index: axis_ok stays in registers
        const bool ok = a == 0 ? axis_ok[0] : (a == 1 ? axis_ok[1] : axis_ok[2]);
        if (!ok) continue;  // warp-uniform
        uint32_t ca;
        float ba[6];
        load(a, ca, ba);
        BinScan s;
        bin_scan(ca, ba, lane, s);
        // lt of candidate i = prefix through bin i-1
        uint32_t lt_cnt = __shfl_up_sync(kFull, s.pre_cnt, 1);
        float lt[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) lt[i] = __shfl_up_sync(kFull, s.pre[i], 1);
        if (lane >= 1 && lane < bins) {
            const uint32_t gt_cnt = s.suf_cnt;
            const float cost =
                split_cost(surface_area6(lt), surface_area6(s.suf), sa_p, lt_cnt, gt_cnt);
            (void)n;
            if (lt_cnt >= P.min_leaf && gt_cnt >= P.min_leaf) {
                const uint64_t k = cand_key(cost, a, lane);
                if (k < best.key) {
                    best.key = k;
                    best.n_lt = lt_cnt;
                    for (int i = 0; i < 6; ++i) {
                        best.lt[i] = lt[i];
                        best.gt[i] = s.suf[i];
                    }
                    best.thr = 0.0f;
                }
            }
        }
    }
}

// The bins held in registers per axis (read by selects: run-time indexes
// into cnt and box would put them in local memory).
__device__ __forceinline__ void binned_candidates(const uint32_t* cnt, const float (*box)[6],
                                                  const bool* axis_ok, uint32_t bins, uint32_t n,
                                                  float sa_p, const Params& P, uint32_t lane,
                                                  Cand& best) {
    binned_candidates_f(
        [&](uint32_t a, uint32_t& ca, float* ba) {
            ca = a == 0 ? cnt[0] : (a == 1 ? cnt[1] : cnt[2]);
#pragma unroll
            for (int i = 0; i < 6; ++i) ba[i] = a == 0 ? box[0][i] : (a == 1 ? box[1][i] : box[2][i]);
        },
        axis_ok, bins, n, sa_p, P, lane, best);
}

// Pull a candidate's payload from lane `src` to all lanes.
__device__ __forceinline__ void shfl_cand(Cand& c, uint32_t src) {
    c.n_lt = __shfl_sync(kFull, c.n_lt, src);
    c.thr = __shfl_sync(kFull, c.thr, src);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        c.lt[i] = __shfl_sync(kFull, c.lt[i], src);
        c.gt[i] = __shfl_sync(kFull, c.gt[i], src);
    }
}

struct XRec {
    float4 lo;  // min xyz, object id (bits)
    float4 hi;  // max xyz, unused
};

// Stable partition of the lanes of segment [s, s+n): lanes with `pred` move
// to the front in lane order, the others follow in lane order. The records
// travel through the warp's exchange area.
__device__ __forceinline__ void warp_stable_permute(bool in_seg, bool pred, uint32_t s, uint32_t n_lt,
                                                    uint32_t lane, float* lo, float* hi,
                                                    uint32_t& id, XRec* x) {
    const uint32_t ltm = __ballot_sync(kFull, in_seg && pred);
    const uint32_t segm = __ballot_sync(kFull, in_seg);
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t dst = pred ? s + __popc(ltm & below) : s + n_lt + __popc(segm & ~ltm & below);
    if (in_seg) {
        x[dst].lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(id));
        x[dst].hi = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
    __syncwarp();
    if (in_seg) {
        const float4 a = x[lane].lo, b = x[lane].hi;
        lo[0] = a.x;
        lo[1] = a.y;
        lo[2] = a.z;
        id = __float_as_uint(a.w);
        hi[0] = b.x;
        hi[1] = b.y;
        hi[2] = b.z;
    }
    __syncwarp();
}

// Build the subtree rooted at a node of n0 <= 32 objects. Lane i < n0 holds
// object i of the node's range (starting at global position `base`).
// Writes every node of the subtree and the permutation entries of its range.
__device__ void warp_build_subtree(float lo[3], float hi[3], uint32_t id, uint32_t n0, uint32_t base,
                                   uint32_t slot0, uint32_t pair0, uint32_t depth0, uint32_t nbase,
                                   uint32_t tbase, const float* bounds0, const Params& P, const Out& O,
                                   XRec* xchg) {
    const uint32_t lane = threadIdx.x & 31u;
    // Pending-node stack, entry k held by lane k.
    uint32_t st_sn = 0, st_slot = 0, st_pair = 0, st_depth = 0;
    float st_b[6];
    if (lane == 0) {
        st_sn = n0 << 8;
        st_slot = slot0;
        st_pair = pair0;
        st_depth = depth0;
        for (int i = 0; i < 6; ++i) st_b[i] = bounds0[i];
    }
    int top = 1;
    uint32_t max_split_depth = 0;
    bool any_split = false;
    uint32_t n_median = 0, n_holes = 0, n_capped = 0;

    while (top > 0) {
        --top;
        const uint32_t sn = __shfl_sync(kFull, st_sn, top);
        const uint32_t s = sn & 0xFFu, n = sn >> 8;
        const uint32_t slot = __shfl_sync(kFull, st_slot, top);
        const uint32_t pair = __shfl_sync(kFull, st_pair, top);
        const uint32_t depth = __shfl_sync(kFull, st_depth, top);
        float nb[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) nb[i] = __shfl_sync(kFull, st_b[i], top);

        const bool in_seg = lane >= s && lane < s + n;
        bool leaf = n <= 1u || depth == P.max_depth ||
                    (n <= P.max_leaf && n < 2u * P.min_leaf);  // bvh/src/lib.rs:548, 556
        uint32_t n_lt = 0;
        Cand win;
        bool adaptive = false;  // adaptive: c < thr; binned: bin < idx; median: position
        bool median = false;
        uint32_t win_axis = 0, win_idx = 0;
        uint32_t mybins = 0;  // this lane's bin per axis (binned sweep), 8 bits each

        if (!leaf) {
            float c[3], cmn[3], cmx[3], ext[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) c[a] = center_of(lo[a], hi[a]);
            // centroid bounds (bvh/src/lib.rs:499-509)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                cmn[a] = funkey(__reduce_min_sync(kFull, in_seg ? fkey(c[a]) : kKeyPosInf));
                cmx[a] = funkey(__reduce_max_sync(kFull, in_seg ? fkey(c[a]) : kKeyNegInf));
                ext[a] = __fsub_rn(cmx[a], cmn[a]);
            }
            const float sa_p = surface_area6(nb);
            Cand best;
            best.key = ~0ull;
            adaptive = n <= P.adaptive_max_n;
            if (adaptive) {
                // adaptive_sweep, bvh/src/lib.rs:392-442
                const bool exact = n < 8u;
                const uint32_t steps =
                    exact ? n : (P.adaptive_steps ? P.adaptive_steps : min(max(n, 8u), 32u));
                const bool cand = exact ? in_seg : lane < steps;
                const uint32_t cidx = exact ? lane - s : lane;
                float thr[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float step = __fdiv_rn(ext[a], __uint2float_rn(steps));
                    thr[a] = exact ? c[a] : adaptive_threshold(cmn[a], step, lane);
                }
                float blt[3][6], bgt[3][6];
                uint32_t nlt[3] = {0, 0, 0};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    box_empty(blt[a]);
                    box_empty(bgt[a]);
                }
                for (uint32_t j = s; j < s + n; ++j) {
                    const float jl0 = __shfl_sync(kFull, lo[0], j), jl1 = __shfl_sync(kFull, lo[1], j),
                                jl2 = __shfl_sync(kFull, lo[2], j);
                    const float jh0 = __shfl_sync(kFull, hi[0], j), jh1 = __shfl_sync(kFull, hi[1], j),
                                jh2 = __shfl_sync(kFull, hi[2], j);
                    const float jc[3] = {center_of(jl0, jh0), center_of(jl1, jh1), center_of(jl2, jh2)};
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        if (jc[a] < thr[a]) {  // bvh/src/lib.rs:308
                            box_grow(blt[a], jl0, jl1, jl2, jh0, jh1, jh2);
                            nlt[a]++;
                        } else {
                            box_grow(bgt[a], jl0, jl1, jl2, jh0, jh1, jh2);
                        }
                    }
                }
                if (cand) {
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const uint32_t ng = n - nlt[a];
                        if (nlt[a] >= P.min_leaf && ng >= P.min_leaf) {  // :407
                            const float cost = split_cost(surface_area6(blt[a]), surface_area6(bgt[a]),
                                                          sa_p, nlt[a], ng);
                            const uint64_t k = cand_key(cost, a, cidx);
                            if (k < best.key) {
                                best.key = k;
                                best.n_lt = nlt[a];
                                best.thr = thr[a];
                                for (int i = 0; i < 6; ++i) {
                                    best.lt[i] = blt[a][i];
                                    best.gt[i] = bgt[a][i];
                                }
                            }
                        }
                    }
                }
            } else {
                // binned_sweep, bvh/src/lib.rs:331-389
                const uint32_t bins = P.bins ? P.bins : min(max(n, 16u), 32u);
                bool axis_ok[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    axis_ok[a] = !(ext[a] == 0.0f);  // :339
                    const uint32_t b = axis_ok[a] ? bin_of(c[a], cmn[a], ext[a], bins) : 0u;
                    mybins |= b << (8 * a);
                }
                uint32_t cnt[3] = {0, 0, 0};
                float box[3][6];
#pragma unroll
                for (int a = 0; a < 3; ++a) box_empty(box[a]);
                for (uint32_t j = s; j < s + n; ++j) {
                    const float jl0 = __shfl_sync(kFull, lo[0], j), jl1 = __shfl_sync(kFull, lo[1], j),
                                jl2 = __shfl_sync(kFull, lo[2], j);
                    const float jh0 = __shfl_sync(kFull, hi[0], j), jh1 = __shfl_sync(kFull, hi[1], j),
                                jh2 = __shfl_sync(kFull, hi[2], j);
                    const uint32_t jb = __shfl_sync(kFull, mybins, j);
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        if (((jb >> (8 * a)) & 0xFFu) == lane) {
                            box_grow(box[a], jl0, jl1, jl2, jh0, jh1, jh2);
                            cnt[a]++;
                        }
                    }
                }
                binned_candidates(cnt, box, axis_ok, bins, n, sa_p, P, lane, best);
            }
            const uint64_t wk = warp_min_key(best.key);
            const uint32_t wlo = static_cast<uint32_t>(wk);
            if (wlo == kNoKey) {
                if (n > P.max_leaf) {
                    median = true;  // bvh/src/lib.rs:527-531
                } else {
                    leaf = true;  // :576-579
                }
            } else {
                win_axis = (wlo >> 8) & 3u;
                win_idx = wlo & 0xFFu;
                const uint32_t src = (adaptive && n < 8u) ? s + win_idx : win_idx;
                win = best;
                shfl_cand(win, src);
                const float cost = funkey(static_cast<uint32_t>(wk >> 32));
                if (n <= P.max_leaf && cost >= leaf_cost(n)) leaf = true;  // :583
                n_lt = win.n_lt;
            }

            if (median) {
                // median_split on axes 0, 1, 2 in turn over the same list
                // (bvh/src/lib.rs:444-491, 528-530); keep the first minimum.
                const uint32_t m = n / 2u;
                uint32_t best_ck = 0;
                for (uint32_t a = 0; a < 3; ++a) {
                    const float ca = center_of(sel3(lo, a), sel3(hi, a));
                    const uint32_t key = fkey(ca);
                    uint32_t rank = 0;
                    for (uint32_t j = s; j < s + n; ++j) {
                        const uint32_t kj = __shfl_sync(kFull, key, j);
                        rank += (kj < key || (kj == key && j < lane)) ? 1u : 0u;
                    }
                    const bool pr = in_seg && rank < m;
                    warp_stable_permute(in_seg, pr, s, m, lane, lo, hi, id, xchg);
                    float blt[6], bgt[6];
                    const bool in_lt = lane >= s && lane < s + m;
                    const bool in_gt = lane >= s + m && lane < s + n;
                    warp_box_union(in_lt, lo, hi, blt);
                    warp_box_union(in_gt, lo, hi, bgt);
                    const float cost =
                        split_cost(surface_area6(blt), surface_area6(bgt), sa_p, m, n - m);
                    const uint32_t ck = fkey(cost);
                    if (a == 0 || ck < best_ck) {
                        best_ck = ck;
                        win_axis = a;
                        for (int i = 0; i < 6; ++i) {
                            win.lt[i] = blt[i];
                            win.gt[i] = bgt[i];
                        }
                    }
                }
                n_lt = m;
                n_median++;
            }
        }

        if (leaf) {
            warp_store_node(O, nbase + slot, nb, base + s - tbase, n, 0u, lane);
            if (in_seg) O.perm[base + lane] = id;
            if (n > 1u) {
                n_holes++;
                if (depth == P.max_depth) n_capped++;
            }
            continue;
        }

        // partition (bvh/src/lib.rs:597-612), stable
        float c[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) c[a] = center_of(lo[a], hi[a]);
        bool pred;
        if (median) {
            pred = lane < s + n_lt;  // Exact { index }: split at the position
        } else if (adaptive) {
            const float cw = win_axis == 0 ? c[0] : (win_axis == 1 ? c[1] : c[2]);
            pred = cw < win.thr;
        } else {
            pred = ((mybins >> (8 * win_axis)) & 0xFFu) < win_idx;
        }
        const uint32_t ltm = __ballot_sync(kFull, in_seg && pred);
        if (static_cast<uint32_t>(__popc(ltm)) != n_lt) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteCount);
        // containment of centroids in child bounds (bvh/src/lib.rs:637-646)
        const bool ok = !in_seg || box_contains2(win.lt, win.gt, pred, c[0], c[1], c[2]);
        if (__ballot_sync(kFull, !ok)) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteContain);
        warp_store_node(O, nbase + slot, nb, base + s - tbase, n, pair, lane);
        if (!median) warp_stable_permute(in_seg, pred, s, n_lt, lane, lo, hi, id, xchg);

        any_split = true;
        max_split_depth = max(max_split_depth, depth);
        const uint32_t n_gt = n - n_lt;
        // push lt, then gt (gt is visited first; order does not change slots)
        if (lane == static_cast<uint32_t>(top)) {
            st_sn = s | (n_lt << 8);
            st_slot = pair + 1u;
            st_pair = pair + 2u * n_gt;
            st_depth = depth + 1u;
            for (int i = 0; i < 6; ++i) st_b[i] = win.lt[i];
        }
        if (lane == static_cast<uint32_t>(top + 1)) {
            st_sn = (s + n_lt) | (n_gt << 8);
            st_slot = pair;
            st_pair = pair + 2u;
            st_depth = depth + 1u;
            for (int i = 0; i < 6; ++i) st_b[i] = win.gt[i];
        }
        top += 2;
    }
    if (lane == 0) {
        if (any_split) atomicMax(&O.ctr->height, max_split_depth);
        if (n_median) atomicAdd(&O.ctr->median_splits, n_median);
        if (n_holes) atomicAdd(&O.ctr->holes, n_holes);
        if (n_capped) atomicAdd(&O.ctr->depth_capped, n_capped);
    }
}

// Segmented reductions over contiguous lane ranges [s, end): shuffle-down
// tree bounded by the segment end, then a broadcast from the segment's first
// lane. Every lane takes part with full masks (per-segment masks in one
// warp serialize: one pass per distinct mask).
__device__ __forceinline__ uint32_t seg_min(uint32_t v, uint32_t lane, uint32_t s, uint32_t end) {
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_down_sync(kFull, v, d);
        if (lane + d < end) v = min(v, u);
    }
    return __shfl_sync(kFull, v, s);
}

__device__ __forceinline__ uint32_t seg_max(uint32_t v, uint32_t lane, uint32_t s, uint32_t end) {
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_down_sync(kFull, v, d);
        if (lane + d < end) v = max(v, u);
    }
    return __shfl_sync(kFull, v, s);
}

// Lexicographic (hi, lo) minimum over the segment.
__device__ __forceinline__ void seg_min2(uint32_t& hi, uint32_t& lo, uint32_t lane, uint32_t s,
                                         uint32_t end) {
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t uh = __shfl_down_sync(kFull, hi, d);
        const uint32_t ul = __shfl_down_sync(kFull, lo, d);
        if (lane + d < end && (uh < hi || (uh == hi && ul < lo))) {
            hi = uh;
            lo = ul;
        }
    }
    hi = __shfl_sync(kFull, hi, s);
    lo = __shfl_sync(kFull, lo, s);
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be scheduled while its predecessor in the stream is
// still finishing. griddepcontrol.wait blocks until the predecessor grid has
// completed and its memory operations are visible (a no-op for an ordinary
// launch); the kernel then lets its own dependent grid be scheduled. Called
// first in every kernel of the build pipeline, before any read of a
// predecessor's output.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Lanes [s, s+n) as a mask.
__device__ __forceinline__ uint32_t seg_mask(uint32_t s, uint32_t n) {
    return n >= 32u ? kFull : (((1u << n) - 1u) << s);
}

// Writes one node from a single lane (two 16-byte stores).
__device__ __forceinline__ void lane_store_node(const Out& o, uint32_t slot, const float* b,
                                                uint32_t start, uint32_t len, uint32_t child) {
    if (slot >= o.node_cap) {
        set_error(o.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
        return;
    }
    float4* p = reinterpret_cast<float4*>(o.nodes + slot);
    p[0] = make_float4(b[0], b[1], b[2], __uint_as_float(start));
    p[1] = make_float4(b[3], b[4], b[5], __uint_as_float(child));
    o.lens[slot] = len;
    o.used[slot] = 1;
}

// Moves this lane's object to lane `dst` (a permutation of the warp).
__device__ __forceinline__ void warp_exchange(uint32_t dst, uint32_t lane, float* lo, float* hi,
                                              uint32_t& id, XRec* x) {
    x[dst].lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(id));
    x[dst].hi = make_float4(hi[0], hi[1], hi[2], 0.0f);
    __syncwarp();
    const float4 a = x[lane].lo, b = x[lane].hi;
    lo[0] = a.x;
    lo[1] = a.y;
    lo[2] = a.z;
    id = __float_as_uint(a.w);
    hi[0] = b.x;
    hi[1] = b.y;
    hi[2] = b.z;
    __syncwarp();
}

// Level-synchronous form of warp_build_subtree: every node of one depth of
// the subtree is evaluated at the same time, each on its own lane range
// (segment), with segmented warp reductions. Valid when every node of the
// subtree uses the adaptive sweep with one threshold per object: the
// reference profile (steps = len.clamp(8,32) = len for 8 <= len <= 32, one
// centroid per object below 8; bvh/src/lib.rs:417-437).
__device__ void warp_build_subtree_levels(float lo[3], float hi[3], uint32_t id, uint32_t n0,
                                          uint32_t base, uint32_t slot0, uint32_t pair0,
                                          uint32_t depth0, uint32_t nbase, uint32_t tbase,
                                          const float* bounds0, const Params& P, const Out& O,
                                          XRec* xchg) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t s = 0, n = n0, slot = slot0, pair = pair0, depth = depth0;
    float nb[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) nb[i] = bounds0[i];
    bool live = lane < n0;
    uint32_t hmax = 0, n_median = 0, n_holes = 0, n_capped = 0;
    bool any_split = false;

    while (__any_sync(kFull, live)) {
        const uint32_t m = live ? seg_mask(s, n) : (1u << lane);
        const uint32_t ss = live ? s : lane, se = live ? s + n : lane + 1u;  // reduction range
        const bool leader = live && lane == s;
        bool leaf = n <= 1u || depth == P.max_depth || (n <= P.max_leaf && n < 2u * P.min_leaf);
        const bool work = live && !leaf;
        float c[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) c[a] = center_of(lo[a], hi[a]);
        const float sa_p = surface_area6(nb);
        const bool exact = n < 8u;
        const uint32_t k = lane - s;
        // thresholds: below 8 objects each object's own centroid; else the
        // adaptive steps over the segment's centroid bounds
        // (bvh/src/lib.rs:499-509), which only such segments need (the
        // warp skips the reductions when it has none)
        float thr[3] = {c[0], c[1], c[2]};
        if (__any_sync(kFull, work && !exact)) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float cmn = funkey(seg_min(work ? fkey(c[a]) : kKeyPosInf, lane, ss, se));
                const float cmx = funkey(seg_max(work ? fkey(c[a]) : kKeyNegInf, lane, ss, se));
                if (!exact) {
                    const float step = __fdiv_rn(__fsub_rn(cmx, cmn), __uint2float_rn(n));
                    thr[a] = adaptive_threshold(cmn, step, k);
                }
            }
        }
        float blt[3][6], bgt[3][6];
        uint32_t nlt[3] = {0, 0, 0};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            box_empty(blt[a]);
            box_empty(bgt[a]);
        }
        const uint32_t maxn = __reduce_max_sync(kFull, work ? n : 0u);
        // every lane's object in shared memory, with its x and y centroids in
        // the spare words; the lanes of a segment read its objects in turn
        // (one address per segment: broadcast loads)
        xchg[lane].lo = make_float4(lo[0], lo[1], lo[2], c[0]);
        xchg[lane].hi = make_float4(hi[0], hi[1], hi[2], c[1]);
        __syncwarp();
        for (uint32_t r = 0; r < maxn; ++r) {
            if (!(work && r < n)) continue;  // lanes past their segment's objects merge nothing
            const float4 ja = xchg[s + r].lo, jb = xchg[s + r].hi;
            const float jl0 = ja.x, jl1 = ja.y, jl2 = ja.z, jh0 = jb.x, jh1 = jb.y, jh2 = jb.z;
            const float jc[3] = {ja.w, jb.w, center_of(jl2, jh2)};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (jc[a] < thr[a]) {  // bvh/src/lib.rs:308
                    blt[a][0] = fminf(blt[a][0], jl0);
                    blt[a][1] = fminf(blt[a][1], jl1);
                    blt[a][2] = fminf(blt[a][2], jl2);
                    blt[a][3] = fmaxf(blt[a][3], jh0);
                    blt[a][4] = fmaxf(blt[a][4], jh1);
                    blt[a][5] = fmaxf(blt[a][5], jh2);
                    nlt[a]++;
                } else {
                    bgt[a][0] = fminf(bgt[a][0], jl0);
                    bgt[a][1] = fminf(bgt[a][1], jl1);
                    bgt[a][2] = fminf(bgt[a][2], jl2);
                    bgt[a][3] = fmaxf(bgt[a][3], jh0);
                    bgt[a][4] = fmaxf(bgt[a][4], jh1);
                    bgt[a][5] = fmaxf(bgt[a][5], jh2);
                }
            }
        }
        __syncwarp();  // reads of xchg done before the exchanges below rewrite it
        Cand best;
        best.key = ~0ull;
        best.n_lt = 0;
        best.thr = 0.0f;
        if (work) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const uint32_t ng = n - nlt[a];
                if (nlt[a] >= P.min_leaf && ng >= P.min_leaf) {  // :407
                    const float cost =
                        split_cost(surface_area6(blt[a]), surface_area6(bgt[a]), sa_p, nlt[a], ng);
                    const uint64_t key = cand_key(cost, a, k);
                    if (key < best.key) {
                        best.key = key;
                        best.n_lt = nlt[a];
                        best.thr = thr[a];
                        for (int i = 0; i < 6; ++i) {
                            best.lt[i] = blt[a][i];
                            best.gt[i] = bgt[a][i];
                        }
                    }
                }
            }
        }
        // first minimum per segment: (cost, axis, threshold index)
        uint32_t mh = static_cast<uint32_t>(best.key >> 32);
        uint32_t ml = static_cast<uint32_t>(best.key);
        seg_min2(mh, ml, lane, ss, se);
        const bool found = work && ml != kNoKey;
        bool median = false;
        uint32_t axis = 0, n_lt = 0;
        Cand win = best;
        shfl_cand(win, found ? s + (ml & 0xFFu) : lane);
        if (work && !found) {
            if (n > P.max_leaf)
                median = true;  // bvh/src/lib.rs:527-531
            else
                leaf = true;  // :576-579
        }
        if (found) {
            axis = (ml >> 8) & 3u;
            n_lt = win.n_lt;
            if (n <= P.max_leaf && funkey(mh) >= leaf_cost(n)) leaf = true;  // :583
        }
        if (__any_sync(kFull, median)) {
            // median_split on axes 0, 1, 2 over the same list (:444-491, :528-530)
            const uint32_t half = n / 2u;
            uint32_t best_ck = 0;
            for (uint32_t a = 0; a < 3; ++a) {
                const uint32_t key = fkey(center_of(sel3(lo, a), sel3(hi, a)));
                uint32_t rank = 0;
                for (uint32_t r = 0; r < maxn; ++r) {
                    const bool use = median && r < n;
                    const uint32_t kj = __shfl_sync(kFull, key, use ? s + r : lane);
                    if (use) rank += (kj < key || (kj == key && s + r < lane)) ? 1u : 0u;
                }
                const bool pr = median && rank < half;
                const uint32_t ltm = __ballot_sync(kFull, pr);
                const uint32_t dst = median ? (pr ? s + __popc(ltm & m & below)
                                                  : s + half + __popc(m & ~ltm & below))
                                            : lane;
                warp_exchange(dst, lane, lo, hi, id, xchg);
                const bool in_lt = median && lane < s + half;
                const bool in_gt = median && lane >= s + half;
                float ml6[6], mg6[6];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    ml6[i] = funkey(seg_min(in_lt ? fkey(lo[i]) : kKeyPosInf, lane, ss, se));
                    mg6[i] = funkey(seg_min(in_gt ? fkey(lo[i]) : kKeyPosInf, lane, ss, se));
                    ml6[3 + i] = funkey(seg_max(in_lt ? fkey(hi[i]) : kKeyNegInf, lane, ss, se));
                    mg6[3 + i] = funkey(seg_max(in_gt ? fkey(hi[i]) : kKeyNegInf, lane, ss, se));
                }
                if (median) {
                    const uint32_t ck =
                        fkey(split_cost(surface_area6(ml6), surface_area6(mg6), sa_p, half, n - half));
                    if (a == 0 || ck < best_ck) {
                        best_ck = ck;
                        axis = a;
                        for (int i = 0; i < 6; ++i) {
                            win.lt[i] = ml6[i];
                            win.gt[i] = mg6[i];
                        }
                    }
                }
            }
            if (median) n_lt = half;
            if (median && leader) n_median++;
        }
        // leaves of this level
        if (live && leaf) {
            if (leader) {
                lane_store_node(O, nbase + slot, nb, base + s - tbase, n, 0u);
                if (n > 1u) {
                    n_holes++;
                    if (depth == P.max_depth) n_capped++;
                }
            }
            O.perm[base + lane] = id;
        }
        const bool split = work && !leaf;
        // partition (bvh/src/lib.rs:597-612), stable; containment (:637-646)
#pragma unroll
        for (int a = 0; a < 3; ++a) c[a] = center_of(lo[a], hi[a]);
        const float ca = axis == 0 ? c[0] : (axis == 1 ? c[1] : c[2]);
        const bool pred = median ? lane < s + n_lt : ca < win.thr;
        const uint32_t ltm = __ballot_sync(kFull, split && pred);
        if (split && lane == s && static_cast<uint32_t>(__popc(ltm & m)) != n_lt)
            set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteCount);
        const bool ok = !split || box_contains2(win.lt, win.gt, pred, c[0], c[1], c[2]);
        if (__any_sync(kFull, !ok) && lane == 0) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteContain);
        if (split && leader) {
            lane_store_node(O, nbase + slot, nb, base + s - tbase, n, pair);
            any_split = true;
            hmax = max(hmax, depth);
        }
        const uint32_t dst =
            split ? (pred ? s + __popc(ltm & m & below) : s + n_lt + __popc(m & ~ltm & below)) : lane;
        warp_exchange(dst, lane, lo, hi, id, xchg);
        if (split) {
            const uint32_t n_gt = n - n_lt;
            if (lane < s + n_lt) {
                n = n_lt;
                slot = pair + 1u;
                pair = pair + 2u * n_gt;
#pragma unroll
                for (int i = 0; i < 6; ++i) nb[i] = win.lt[i];
            } else {
                s = s + n_lt;
                n = n_gt;
                slot = pair;
                pair = pair + 2u;
#pragma unroll
                for (int i = 0; i < 6; ++i) nb[i] = win.gt[i];
            }
            depth++;
            // a child that the leaf rule stops (:556) is written now rather
            // than by one more pass of the loop (the same node and entries)
            if (n <= 1u || depth == P.max_depth || (n <= P.max_leaf && n < 2u * P.min_leaf)) {
                if (lane == s) {
                    lane_store_node(O, nbase + slot, nb, base + s - tbase, n, 0u);
                    if (n > 1u) {
                        n_holes++;
                        if (depth == P.max_depth) n_capped++;
                    }
                }
                O.perm[base + lane] = id;
                live = false;
            }
        }
        if (leaf) live = false;
    }
    // counters: one atomic per warp
    const uint32_t hm = __reduce_max_sync(kFull, any_split ? hmax : 0u);
    const bool anys = __any_sync(kFull, any_split);
    const uint32_t med = __reduce_add_sync(kFull, n_median);
    const uint32_t hol = __reduce_add_sync(kFull, n_holes);
    const uint32_t cap = __reduce_add_sync(kFull, n_capped);
    if (lane == 0) {
        if (anys) atomicMax(&O.ctr->height, hm);
        if (med) atomicAdd(&O.ctr->median_splits, med);
        if (hol) atomicAdd(&O.ctr->holes, hol);
        if (cap) atomicAdd(&O.ctr->depth_capped, cap);
    }
}

}  // namespace mgbvh
