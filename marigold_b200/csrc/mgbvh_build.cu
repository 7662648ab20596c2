// mgbvh_build.cu — B200 SAH BVH builder: kernels, orchestration and C ABI.
//
// The tree is the one bvh/src/lib.rs:698-878 builds, bit for bit: same split
// decisions, node bounds, child links, start indices and (for single-object
// leaves) object order. Work is split by node size:
//
//   large  (len > kMediumMax)   level-synchronous over all large nodes:
//                               lvl_bin   per-tile 3x32-bin histograms of
//                                         counts and AABBs in shared memory,
//                                         merged across tiles with atomics
//                               lvl_eval  one warp per node: prefix/suffix
//                                         sweeps, SAH costs, argmin, children
//                               lvl_part  stable scan partition of the
//                                         node's 32-byte object records
//   medium (33..kMediumMax)     one CTA per node builds the whole subtree
//                               with records in shared memory, warps per
//                               sub-node, 16-bit index partitions
//   small  (<= 32)              one warp per subtree, objects in registers
//                               (mgbvh_device.cuh)
//
// Node slots come from the closed-form pre-order numbering (see Out in
// mgbvh_device.cuh); a compaction pass removes holes left by multi-object
// leaves.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "mgbvh_device.cuh"
#include "mgbvh_learn.cuh"

namespace mgbvh {

constexpr uint32_t kMediumMax = 1024;
#ifndef MGBVH_TILE
#define MGBVH_TILE 2048  // objects per level-pass tile (tuning knob; a multiple of 256 * the bin batch)
#endif
constexpr uint32_t kTile = MGBVH_TILE;
constexpr int kTileThreads = 256;
#ifndef MGBVH_MEDIUM_WARPS
#define MGBVH_MEDIUM_WARPS 4  // warps per subtree CTA (tuning knob)
#endif
#ifndef MGBVH_MEDIUM_SMALL_CTAS
#define MGBVH_MEDIUM_SMALL_CTAS 5  // CTAs per SM of the 512-object instance (tuning knob)
#endif
constexpr int kMediumWarps = MGBVH_MEDIUM_WARPS;
constexpr int kMediumThreads = kMediumWarps * 32;
constexpr uint32_t kBinWords = 3 * 32 * 7;  // [axis][bin]{count, lo key xyz, hi key xyz}

// Level counter slots rotate over three: level L reads ctr->lvl[L % 3],
// its evaluations append the next level's nodes to slot (L + 1) % 3, and
// slot (L + 2) % 3, last read by level L - 1, is cleared during level L.
__host__ __device__ __forceinline__ uint32_t lvl_next(uint32_t lv) { return lv == 2u ? 0u : lv + 1u; }
__host__ __device__ __forceinline__ uint32_t lvl_free(uint32_t lv) { return lv == 0u ? 2u : lv - 1u; }
constexpr uint32_t kNone = 0xFFFFFFFFu;

struct Rec {
    float4 lo;  // min xyz, object id (bits)
    float4 hi;  // max xyz, 0
};

// A record read through L2 only. Within one launch of the persistent batched
// build, records are rewritten by other CTAs (other SMs), whose writes an
// SM's L1 does not see: reads of such data bypass L1.
__device__ __forceinline__ Rec ldcg_rec(const Rec* p) {
    Rec r;
    r.lo = __ldcg(&p->lo);
    r.hi = __ldcg(&p->hi);
    return r;
}

template <bool kCoherent>
__device__ __forceinline__ Rec load_rec(const Rec* p) {
    if constexpr (kCoherent)
        return ldcg_rec(p);
    else
        return *p;
}

// A node waiting to be split (large, medium or small list entry). 64 bytes.
struct Task {
    float lo[3];
    uint32_t start;
    float hi[3];
    uint32_t len;
    uint32_t slot, pair, depth, buf;
    uint32_t tile0, ntiles;
    uint32_t nbase, tbase;  // node-slot and record offsets of the object's mesh (batched builds)
};

// A task read through L2 only (see ldcg_rec).
__device__ __forceinline__ Task ldcg_task(const Task* p) {
    static_assert(sizeof(Task) == 64, "task layout");
    Task t;
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4* d = reinterpret_cast<uint4*>(&t);
#pragma unroll
    for (int k = 0; k < 4; ++k) d[k] = __ldcg(q + k);
    return t;
}

// Split decision of one large node, read by its partition tiles.
struct Decision {
    uint32_t kind;  // 0 split, 1 leaf (or a forced median deferred to the median passes)
    uint32_t axis, split_bin, bins;
    float cmin, ext;
    uint32_t n_lt;
    uint32_t child_task[2];  // [0] gt, [1] lt: next-level large task, or kNone
    uint32_t child_leaf[2];
    uint32_t use_thr;    // 1: a learned proposal won; the partition is centroid < thr
    float thr;
    uint32_t plain_key;  // cost key of the binned split
    float ltb[6], gtb[6];
};

// ---------------------------------------------------------------- helpers

// Grows the lt (k[0..5]: min keys xyz, max keys xyz) or gt (k[6..11])
// centroid key bounds by centroid c; selects with constant indexes keep k in
// registers.
__device__ __forceinline__ void grow_keys12(uint32_t* k, bool lt, const float* c) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const uint32_t f = fkey(c[a]);
        k[a] = lt ? min(k[a], f) : k[a];
        k[3 + a] = lt ? max(k[3 + a], f) : k[3 + a];
        k[6 + a] = lt ? k[6 + a] : min(k[6 + a], f);
        k[9 + a] = lt ? k[9 + a] : max(k[9 + a], f);
    }
}

__device__ __forceinline__ void block_reduce_keys_to_global(uint32_t* keys /*12*/, uint32_t* smem12,
                                                            uint32_t* global12) {
    // keys[0..5]: min keys; keys[6..11] : max keys ; layout per call site
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
        const bool is_min = (k % 6) < 3;
        const uint32_t v = is_min ? __reduce_min_sync(kFull, keys[k]) : __reduce_max_sync(kFull, keys[k]);
        if (lane == 0) {
            if (is_min)
                atomicMin(&smem12[k], v);
            else
                atomicMax(&smem12[k], v);
        }
    }
    __syncthreads();
    if (threadIdx.x < 12) {
        const bool is_min = (threadIdx.x % 6) < 3;
        if (is_min)
            atomicMin(&global12[threadIdx.x], smem12[threadIdx.x]);
        else
            atomicMax(&global12[threadIdx.x], smem12[threadIdx.x]);
    }
}

__device__ __forceinline__ void init_key12(uint32_t* k) {
#pragma unroll
    for (int i = 0; i < 12; ++i) k[i] = ((i % 6) < 3) ? kKeyPosInf : kKeyNegInf;
}

__device__ __forceinline__ void accum_keys(uint32_t* k, float lx, float ly, float lz, float hx,
                                           float hy, float hz) {
    // bounds: k[0..2] min lo, k[3..5] max hi; centroids: k[6..8] min, k[9..11] max
    k[0] = min(k[0], fkey(lx));
    k[1] = min(k[1], fkey(ly));
    k[2] = min(k[2], fkey(lz));
    k[3] = max(k[3], fkey(hx));
    k[4] = max(k[4], fkey(hy));
    k[5] = max(k[5], fkey(hz));
    const uint32_t c0 = fkey(center_of(lx, hx)), c1 = fkey(center_of(ly, hy)),
                   c2 = fkey(center_of(lz, hz));
    k[6] = min(k[6], c0);
    k[7] = min(k[7], c1);
    k[8] = min(k[8], c2);
    k[9] = max(k[9], c0);
    k[10] = max(k[10], c1);
    k[11] = max(k[11], c2);
}

// ---------------------------------------------------------------- prep

// Object records from MeshTriangle/MeshVertex (mesh_interface/src/lib.rs:19-30)
// plus the root's bounds and centroid bounds.
__global__ void __launch_bounds__(256) prep_indexed_kernel(const float* __restrict__ verts,
                                                           uint32_t stride_floats, uint32_t nverts,
                                                           const uint32_t* __restrict__ tris,
                                                           uint32_t n, Rec* __restrict__ out,
                                                           Counters* ctr) {
    pdl_enter();
    __shared__ uint32_t sk[12];
    if (threadIdx.x < 12) sk[threadIdx.x] = ((threadIdx.x % 6) < 3) ? kKeyPosInf : kKeyNegInf;
    __syncthreads();
    uint32_t k[12];
    init_key12(k);
    const bool vec4 = (stride_floats & 3u) == 0u && (reinterpret_cast<uintptr_t>(verts) & 15u) == 0u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t t0 = tris[3 * (size_t)i], t1 = tris[3 * (size_t)i + 1], t2 = tris[3 * (size_t)i + 2];
        if (t0 >= nverts || t1 >= nverts || t2 >= nverts) {
            set_error(ctr, MGBVH_ERR_INVALID_ARG, kSiteIndex);
            t0 = t1 = t2 = 0;
        }
        const float* p0 = verts + (size_t)t0 * stride_floats;
        const float* p1 = verts + (size_t)t1 * stride_floats;
        const float* p2 = verts + (size_t)t2 * stride_floats;
        float v0[3], v1[3], v2[3];
        if (vec4) {
            // 16-byte vertex rows: one load per vertex (the position and
            // the next word of the row, which is not used)
            const float4 a = __ldg(reinterpret_cast<const float4*>(p0));
            const float4 b = __ldg(reinterpret_cast<const float4*>(p1));
            const float4 c = __ldg(reinterpret_cast<const float4*>(p2));
            v0[0] = a.x, v0[1] = a.y, v0[2] = a.z;
            v1[0] = b.x, v1[1] = b.y, v1[2] = b.z;
            v2[0] = c.x, v2[1] = c.y, v2[2] = c.z;
        } else {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                v0[q] = __ldg(p0 + q);
                v1[q] = __ldg(p1 + q);
                v2[q] = __ldg(p2 + q);
            }
        }
        float lo[3], hi[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float x0 = __fadd_rn(v0[a], 0.0f), x1 = __fadd_rn(v1[a], 0.0f), x2 = __fadd_rn(v2[a], 0.0f);
            lo[a] = fminf(fminf(x0, x1), x2);
            hi[a] = fmaxf(fmaxf(x0, x1), x2);
        }
        Rec r;
        r.lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(i));
        r.hi = make_float4(hi[0], hi[1], hi[2], 0.0f);
        out[i] = r;
        accum_keys(k, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
    }
    block_reduce_keys_to_global(k, sk, ctr->root_keys);
}

// Object records from AABBs (min xyz, max xyz): the AsBoundingVolume path.
__global__ void __launch_bounds__(256) prep_aabbs_kernel(const float* __restrict__ aabbs, uint32_t n,
                                                         Rec* __restrict__ out, Counters* ctr) {
    pdl_enter();
    __shared__ uint32_t sk[12];
    if (threadIdx.x < 12) sk[threadIdx.x] = ((threadIdx.x % 6) < 3) ? kKeyPosInf : kKeyNegInf;
    __syncthreads();
    uint32_t k[12];
    init_key12(k);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* p = aabbs + 6 * (size_t)i;
        float v[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) v[j] = __fadd_rn(__ldg(p + j), 0.0f);
        Rec r;
        r.lo = make_float4(v[0], v[1], v[2], __uint_as_float(i));
        r.hi = make_float4(v[3], v[4], v[5], 0.0f);
        out[i] = r;
        accum_keys(k, v[0], v[1], v[2], v[3], v[4], v[5]);
    }
    block_reduce_keys_to_global(k, sk, ctr->root_keys);
}

__device__ __forceinline__ void init_task_bins(uint32_t* b, uint32_t lane, uint32_t nthreads) {
    for (uint32_t w = lane; w < kBinWords; w += nthreads) {
        const uint32_t f = w % 7u;
        b[w] = f == 0 ? 0u : (f <= 3 ? kKeyPosInf : kKeyNegInf);
    }
}

// Root node: classify and enqueue (or finish, when the root is a leaf).
// cls: 0 leaf, 1 small, 2 medium, 3 large.
__global__ void init_root_kernel(uint32_t n, uint32_t cls, uint32_t has_bounds, float b0, float b1,
                                 float b2, float b3, float b4, float b5, Task* large, uint32_t* bins,
                                 uint32_t* cbkeys, uint32_t* tile_task, uint32_t* tile_begin,
                                 Task* medium, Task* small, Out O, uint32_t ntiles,
                                 uint32_t max_depth) {
    pdl_enter();
    float b[6];
    if (has_bounds) {
        b[0] = b0; b[1] = b1; b[2] = b2; b[3] = b3; b[4] = b4; b[5] = b5;
    } else {
        for (int i = 0; i < 6; ++i) b[i] = funkey(O.ctr->root_keys[i]);
    }
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gsz = gridDim.x * blockDim.x;
    Task t;
    for (int a = 0; a < 3; ++a) {
        t.lo[a] = b[a];
        t.hi[a] = b[3 + a];
    }
    t.start = 0;
    t.len = n;
    t.slot = 0;
    t.pair = 1;
    t.depth = 0;
    t.buf = 0;
    t.tile0 = 0;
    t.ntiles = ntiles;
    t.nbase = t.tbase = 0;
    if (cls == 0) {
        if (gtid == 0) {
            mgbvh_node nd;
            for (int a = 0; a < 3; ++a) {
                nd.min[a] = b[a];
                nd.max[a] = b[3 + a];
            }
            nd.start_index = 0;
            nd.child_node = 0;
            O.nodes[0] = nd;
            O.lens[0] = n;
            O.used[0] = 1;
            if (n > 1) {
                atomicAdd(&O.ctr->holes, 1u);
                if (max_depth == 0) atomicAdd(&O.ctr->depth_capped, 1u);
            }
        }
        for (uint32_t i = gtid; i < n; i += gsz) O.perm[i] = i;
        return;
    }
    if (cls == 1) {
        if (gtid == 0) {
            small[0] = t;
            O.ctr->n_small = 1;
        }
        return;
    }
    if (cls == 2) {
        if (gtid == 0) {
            medium[0] = t;
            O.ctr->n_medium = 1;
        }
        return;
    }
    if (gtid == 0) {
        large[0] = t;
        O.ctr->lvl[0][0] = 1;
        O.ctr->lvl[0][1] = ntiles;
    }
    if (blockIdx.x == 0) init_task_bins(bins, threadIdx.x, blockDim.x);
    if (gtid < 6) cbkeys[gtid] = O.ctr->root_keys[6 + gtid];
    for (uint32_t i = gtid; i < ntiles; i += gsz) {
        tile_task[i] = 0;
        tile_begin[i] = i * kTile;
    }
}

// ---------------------------------------------------------------- large level

constexpr uint32_t kRecsPerThread = kTile / kTileThreads;  // 8


#ifndef MGBVH_BIN_MIN_BLOCKS
#define MGBVH_BIN_MIN_BLOCKS 4  // CTAs per SM the register budget must allow (tuning knob; 1 / 3 / 4 with batches of 8 / 4 / 4: 682 / 691 / 692 Mtri/s)
#endif
#ifndef MGBVH_PART_CODES
#define MGBVH_PART_CODES 1  // 1: the bin pass stores each record's bins (16 bits) and the partition reads them
#endif
constexpr bool kPartCodes = MGBVH_PART_CODES != 0;
#ifndef MGBVH_BIN_BATCH
#define MGBVH_BIN_BATCH 4  // records a thread loads before binning them (tuning knob; divides 8)
#endif
constexpr uint32_t kBinBatch = MGBVH_BIN_BATCH;
static_assert(kRecsPerThread % kBinBatch == 0, "the bin batch divides the records per thread");
#ifndef MGBVH_PART_UNROLL
#define MGBVH_PART_UNROLL 1  // records in flight per lane in the scatter pass (tuning knob; 1 / 2 / 4: 681 / 676 / 680 Mtri/s)
#endif
constexpr int kPartUnroll = MGBVH_PART_UNROLL;


struct EvalArgs {
    const Task* tasks;
    uint32_t lv;  // level counter slot: counts in ctr->lvl[lv], next level's in ctr->lvl[lvl_next(lv)]
    const uint32_t* bins;
    const uint32_t* cbkeys;
    const uint32_t* tile_hist;  // [axis * 32 + bin][tile]: objects of the tile in the axis's bins below bin
    uint32_t* tile_lt;
    Decision* dec;
    Task* next_tasks;
    uint32_t* next_bins;
    uint32_t* next_cbkeys;
    uint32_t* next_tile_task;
    uint32_t* next_tile_begin;
    Task* medium;
    Task* small;
    uint32_t cap_tasks, cap_tiles, cap_medium, cap_small;
    // learned form (lw NULL: off): transposed network parameters, refine gate,
    // per-task pending proposals, their interval bins and per-tile counts
    const __nv_bfloat16* lw;
    int lgate;
    float lgate_thr;  // refine-logit threshold of the gate
    uint32_t lmin_n;  // smallest node that runs the network
    LvlRefine* refine;
    uint32_t* rbins;
    const uint32_t* tile_hist2;  // [proposal * 17 + interval][tile]: objects in intervals 0..interval
    Task* med;  // nodes waiting for a forced median (cap_tasks entries; count in ctr->n_med)
};

// Writes the node and its children of a decided split: the per-tile lt
// counts (exclusive scan across the node's tiles of histogram row `row`:
// each tile's objects left of the split), the node record, and each child as
// a leaf, a next-level task, a medium or a small subtree. Each lane scans a
// contiguous run of the node's tiles (independent loads), runs joined by a
// warp scan.
__device__ void emit_split(const EvalArgs& A, const Params& P, const Out& O, uint32_t w, uint32_t lane,
                           const Task& t, Decision& d, const uint32_t* hist, uint32_t row) {
    const float nb[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
    const uint32_t* h = hist + (size_t)row * A.cap_tiles + t.tile0;
    uint32_t* lt = A.tile_lt + t.tile0;
    const uint32_t per = (t.ntiles + 31u) >> 5;
    const uint32_t i0 = min(lane * per, t.ntiles), i1 = min(i0 + per, t.ntiles);
    uint32_t sum = 0;
#pragma unroll 8
    for (uint32_t i = i0; i < i1; ++i) sum += h[i];
    uint32_t inc = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, inc, off);
        if (lane >= static_cast<uint32_t>(off)) inc += u;
    }
    const uint32_t total = __shfl_sync(kFull, inc, 31);
    uint32_t run = inc - sum;
    for (uint32_t i = i0; i < i1; ++i) {
        const uint32_t v = h[i];
        lt[i] = run;
        run += v;
    }
    if (total != d.n_lt && lane == 0) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteCount);
    warp_store_node(O, t.nbase + t.slot, nb, t.start - t.tbase, t.len, t.pair, lane);
    if (lane == 0) atomicMax(&O.ctr->height, t.depth);
    const uint32_t n_gt = t.len - d.n_lt;
    // each child's class (0 leaf, 1 next-level task, 2 medium, 3 small), then
    // one atomic per list for both children
    uint32_t cls[2], ntl[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const uint32_t len = c == 0 ? n_gt : d.n_lt;
        const uint32_t depth = t.depth + 1u;
        const bool cleaf = len <= 1u || depth == P.max_depth || (len <= P.max_leaf && len < 2u * P.min_leaf);
        cls[c] = cleaf ? 0u : (len > P.medium_max ? 1u : (len > kSmallMax ? 2u : 3u));
        ntl[c] = cls[c] == 1u ? (len + kTile - 1) / kTile : 0u;
    }
    uint32_t slot_task = 0, slot_tile = 0, slot_med = 0, slot_small = 0;
    if (lane == 0) {
        const uint32_t nl = (cls[0] == 1u) + (cls[1] == 1u), nm = (cls[0] == 2u) + (cls[1] == 2u),
                       ns = (cls[0] == 3u) + (cls[1] == 3u);
        if (nl) {
            slot_task = atomicAdd(&O.ctr->lvl[lvl_next(A.lv)][0], nl);
            slot_tile = atomicAdd(&O.ctr->lvl[lvl_next(A.lv)][1], ntl[0] + ntl[1]);
        }
        if (nm) slot_med = atomicAdd(&O.ctr->n_medium, nm);
        if (ns) slot_small = atomicAdd(&O.ctr->n_small, ns);
    }
    slot_task = __shfl_sync(kFull, slot_task, 0);
    slot_tile = __shfl_sync(kFull, slot_tile, 0);
    slot_med = __shfl_sync(kFull, slot_med, 0);
    slot_small = __shfl_sync(kFull, slot_small, 0);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const uint32_t len = c == 0 ? n_gt : d.n_lt;
        const uint32_t start = c == 0 ? t.start + d.n_lt : t.start;
        const uint32_t slot = c == 0 ? t.pair : t.pair + 1u;
        const uint32_t pair = c == 0 ? t.pair + 2u : t.pair + 2u * n_gt;
        const uint32_t depth = t.depth + 1u;
        const float* cb = c == 0 ? d.gtb : d.ltb;
        Task ct;
        for (int a = 0; a < 3; ++a) {
            ct.lo[a] = cb[a];
            ct.hi[a] = cb[3 + a];
        }
        ct.start = start;
        ct.len = len;
        ct.slot = slot;
        ct.pair = pair;
        ct.depth = depth;
        ct.buf = t.buf ^ 1u;
        ct.tile0 = ct.ntiles = 0;
        ct.nbase = t.nbase;
        ct.tbase = t.tbase;
        // this child's place in its list: after the gt child when both share it
        const uint32_t before = (c == 1 && cls[0] == cls[1]) ? 1u : 0u;
        if (cls[c] == 0u) {
            warp_store_node(O, t.nbase + slot, cb, start - t.tbase, len, 0u, lane);
            d.child_leaf[c] = 1;
            if (lane == 0 && len > 1) {
                atomicAdd(&O.ctr->holes, 1u);
                if (depth == P.max_depth) atomicAdd(&O.ctr->depth_capped, 1u);
            }
        } else if (cls[c] == 1u) {
            const uint32_t nt = ntl[c];
            const uint32_t ti = slot_task + before;
            const uint32_t t0 = slot_tile + (c == 1 && cls[0] == 1u ? ntl[0] : 0u);
            if (ti >= A.cap_tasks || t0 + nt > A.cap_tiles) {
                if (lane == 0) set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                continue;
            }
            ct.tile0 = t0;
            ct.ntiles = nt;
            if (lane == 0) A.next_tasks[ti] = ct;
            init_task_bins(A.next_bins + (size_t)ti * kBinWords, lane, 32);
            if (lane < 6) A.next_cbkeys[6 * ti + lane] = lane < 3 ? kKeyPosInf : kKeyNegInf;
            for (uint32_t i = lane; i < nt; i += 32) {
                A.next_tile_task[t0 + i] = ti;
                A.next_tile_begin[t0 + i] = i * kTile;
            }
            d.child_task[c] = ti;
        } else if (cls[c] == 2u) {
            const uint32_t mi = slot_med + before;
            if (mi >= A.cap_medium) {
                if (lane == 0) set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                continue;
            }
            if (lane == 0) A.medium[mi] = ct;
        } else {
            const uint32_t si = slot_small + before;
            if (si >= A.cap_small) {
                if (lane == 0) set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                continue;
            }
            if (lane == 0) A.small[si] = ct;
        }
    }
    if (lane == 0) A.dec[w] = d;
}

// transposed network parameters as 16-byte vectors (the learned evaluation
// stages them in shared memory)
constexpr uint32_t kEvalWeightVec = mgbvh_mlp::kTParams * 2u / 16u;
static_assert(mgbvh_mlp::kTParams * 2u % 16u == 0u, "the transposed parameters are whole 16-byte vectors");
constexpr size_t kEvalWeightBytes = mgbvh_mlp::kTParams * 2u;

// kLearn: with the learned form's network (a separate instantiation keeps
// the plain evaluation's code small: a cold kernel fetches every instruction).
template <bool kLearn>
__device__ void eval_task(const EvalArgs& A, const Params& P, const Out& O, uint32_t w, uint32_t lane) {
    const Task t = A.tasks[w];
    const uint32_t* tb = A.bins + (size_t)w * kBinWords;
    if (A.refine && lane == 0) A.refine[w].on = 0;  // before any return: nothing pending
    float cmn[3], ext[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        cmn[a] = funkey(A.cbkeys[6 * w + a]);
        ext[a] = __fsub_rn(funkey(A.cbkeys[6 * w + 3 + a]), cmn[a]);
    }
    const float nb[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
    const uint32_t B = P.bins ? P.bins : 32u;
    bool leaf = t.depth == P.max_depth || (t.len <= P.max_leaf && t.len < 2u * P.min_leaf);
    Decision d;
    d.kind = 1;
    d.axis = d.split_bin = 0;
    d.bins = B;
    d.cmin = d.ext = 0.0f;
    d.n_lt = 0;
    d.child_task[0] = d.child_task[1] = kNone;
    d.child_leaf[0] = d.child_leaf[1] = 0;
    d.use_thr = 0;
    d.thr = 0.0f;
    d.plain_key = kNoKey;
    Cand win;
    uint32_t cnt[3] = {0, 0, 0};
    if (!leaf) {
        float box[3][6];
        bool axis_ok[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const uint32_t* bw = tb + (a * 32 + lane) * 7;
            cnt[a] = bw[0];
            for (int i = 0; i < 6; ++i) box[a][i] = funkey(bw[1 + i]);
            axis_ok[a] = !(ext[a] == 0.0f);
        }
        Cand best;
        binned_candidates(cnt, box, axis_ok, B, t.len, surface_area6(nb), P, lane, best);
        const uint64_t wk = warp_min_key(best.key);
        const uint32_t wlo = static_cast<uint32_t>(wk);
        if (wlo == kNoKey) {
            if (t.len > P.max_leaf) {
                // no binned split and too many objects for a leaf: the forced
                // median (bvh/src/lib.rs:527-531) runs in the median passes
                // after this build's pipeline. The partition treats the node
                // as a leaf: it only copies the ids into the permutation, which
                // the leaves of the node's subtree overwrite later.
                if (lane == 0) {
                    d.kind = 1;
                    A.dec[w] = d;
                    const uint32_t mi = atomicAdd(&O.ctr->n_med, 1u);
                    if (mi < A.cap_tasks)
                        A.med[mi] = t;
                    else
                        set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                }
                return;
            }
            leaf = true;
        } else {
            d.axis = (wlo >> 8) & 3u;
            d.split_bin = wlo & 0xFFu;
            d.plain_key = static_cast<uint32_t>(wk >> 32);
            win = best;
            shfl_cand(win, d.split_bin);
            const float cost = funkey(d.plain_key);
            if (t.len <= P.max_leaf && cost >= leaf_cost(t.len)) leaf = true;
        }
    }
    if (leaf) {
        warp_store_node(O, t.nbase + t.slot, nb, t.start - t.tbase, t.len, 0u, lane);
        if (lane == 0) {
            A.dec[w] = d;
            if (t.len > 1) {
                atomicAdd(&O.ctr->holes, 1u);
                if (t.depth == P.max_depth) atomicAdd(&O.ctr->depth_capped, 1u);
            }
        }
        return;
    }
    d.kind = 0;
    d.cmin = sel3(cmn, d.axis);
    d.ext = sel3(ext, d.axis);
    d.n_lt = win.n_lt;
    for (int i = 0; i < 6; ++i) {
        d.ltb[i] = win.lt[i];
        d.gtb[i] = win.gt[i];
    }
    if (kLearn && A.lw && B == 32u && t.len >= A.lmin_n) {
        // the learned form: run the network; with proposals to score, the
        // decision waits for the refine pass (lvl_eval2_kernel)
        const float cb[6] = {cmn[0], cmn[1], cmn[2], funkey(A.cbkeys[6 * w + 3]),
                             funkey(A.cbkeys[6 * w + 4]), funkey(A.cbkeys[6 * w + 5])};
        float f[24];
        node_features(nb, cb, t.len, t.depth, cnt, f);
        int top0 = 0, top1 = 0;
        float refine = 0.0f;
        mgbvh_mlp::warp_forward_t(f, A.lw, lane, top0, top1, refine);
        const bool on = !A.lgate || refine > A.lgate_thr;
        if (lane == 0) {
            LvlRefine R;
            R.on = on ? 1u : 0u;
            R.prop[0] = (uint32_t)top0;
            R.prop[1] = (uint32_t)top1;
            R.pad = 0;
            A.refine[w] = R;
        }
        if (on) {
            uint32_t* rb = A.rbins + (size_t)w * kRBinWords;
            for (uint32_t i = lane; i < kRBinWords; i += 32) {
                const uint32_t f7 = i % 7u;
                rb[i] = f7 == 0 ? 0u : (f7 <= 3 ? kKeyPosInf : kKeyNegInf);
            }
            if (lane == 0) A.dec[w] = d;
            return;
        }
    }
    emit_split(A, P, O, w, lane, t, d, A.tile_hist, d.axis * 32u + d.split_bin);
}

template <bool kLearn>
__global__ void __launch_bounds__(128) lvl_eval_kernel(EvalArgs A, Params P, Out O) {
    pdl_enter();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n_tasks = O.ctr->lvl[A.lv][0];
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    if constexpr (kLearn) {
        // the network's parameters staged in shared memory by the whole CTA
        // (19.8 KB, coalesced), so each forward pass reads them at shared-memory
        // latency instead of one dependent L2 round trip per group of inputs
        extern __shared__ __align__(16) unsigned char eval_dsm[];
        if (blockIdx.x * (blockDim.x >> 5) >= n_tasks) return;  // block-uniform: no node here
        if (A.lw) {
            const uint4* gw = reinterpret_cast<const uint4*>(A.lw);
            uint4* sw = reinterpret_cast<uint4*>(eval_dsm);
            for (uint32_t i = threadIdx.x; i < kEvalWeightVec; i += blockDim.x) sw[i] = gw[i];
            __syncthreads();
            A.lw = reinterpret_cast<const __nv_bfloat16*>(eval_dsm);
        }
    }
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_tasks; w += nwarps)
        eval_task<kLearn>(A, P, O, w, lane);
}

// Per-tile bin histograms (count + AABB per axis and bin) of the large nodes
// with shared-memory atomics, merged into the node's global bins. Grid-stride over
// the level's tiles; the tile count is read on the device. Each thread loads
// its records of the tile first (kTile / kTileThreads of them), then bins
// them. Also clears the level counter slot two levels ahead (the previous
// level's kernels, which read it, have finished; the next writer is the
// next level's evaluation). Each record's bin on every axis (5 bits each)
// goes to `codes` at its position, for the partition pass.
__global__ void __launch_bounds__(kTileThreads, MGBVH_BIN_MIN_BLOCKS) lvl_bin_kernel(
    const Task* __restrict__ tasks, const uint32_t* __restrict__ cbkeys, uint32_t* __restrict__ bins,
    const uint32_t* __restrict__ tile_task, const uint32_t* __restrict__ tile_begin,
    uint32_t* __restrict__ tile_hist, uint32_t cap_tiles, const Rec* __restrict__ rec0,
    const Rec* __restrict__ rec1, uint16_t* __restrict__ codes, Counters* __restrict__ ctr, uint32_t lv,
    Params P) {
    pdl_enter();
    __shared__ uint32_t sb[kBinWords];
    if (blockIdx.x == 0 && threadIdx.x < 2) ctr->lvl[lvl_free(lv)][threadIdx.x] = 0;
    const uint32_t ntiles = ctr->lvl[lv][1];
    const uint32_t B = P.bins ? P.bins : 32u;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        __syncthreads();
        init_task_bins(sb, threadIdx.x, blockDim.x);
        const uint32_t ti = tile_task[tile];
        const Task& t = tasks[ti];
        const uint32_t begin = tile_begin[tile];
        const uint32_t cnt = min(kTile, t.len - begin);
        const Rec* src = (t.buf ? rec1 : rec0) + t.start + begin;
        float cmn[3], ext[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            cmn[a] = funkey(cbkeys[6 * ti + a]);
            ext[a] = __fsub_rn(funkey(cbkeys[6 * ti + 3 + a]), cmn[a]);
        }
        // records loaded kBinBatch at a time, then binned
#pragma unroll
        for (uint32_t k0 = 0; k0 < kRecsPerThread; k0 += kBinBatch) {
            float4 rl[kBinBatch], rh[kBinBatch];
#pragma unroll
            for (uint32_t k = 0; k < kBinBatch; ++k) {
                const uint32_t i = threadIdx.x + (k0 + k) * kTileThreads;
                if (i < cnt) {
                    rl[k] = src[i].lo;
                    rh[k] = src[i].hi;
                }
            }
            if (k0 == 0) __syncthreads();  // the tile's bins are initialized
#pragma unroll
            for (uint32_t k = 0; k < kBinBatch; ++k) {
                const uint32_t i = threadIdx.x + (k0 + k) * kTileThreads;
                if (i >= cnt) break;
                const float l[3] = {rl[k].x, rl[k].y, rl[k].z}, h[3] = {rh[k].x, rh[k].y, rh[k].z};
                uint32_t code = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    if (ext[a] == 0.0f) continue;  // block-uniform
                    const uint32_t b = bin_of(center_of(l[a], h[a]), cmn[a], ext[a], B);
                    code |= b << (5 * a);
                    uint32_t* w = sb + (a * 32 + b) * 7;
                    atomicAdd(w, 1u);
                    atomicMin(w + 1, fkey(l[0]));
                    atomicMin(w + 2, fkey(l[1]));
                    atomicMin(w + 3, fkey(l[2]));
                    atomicMax(w + 4, fkey(h[0]));
                    atomicMax(w + 5, fkey(h[1]));
                    atomicMax(w + 6, fkey(h[2]));
                }
                if (kPartCodes) codes[t.start + begin + i] = static_cast<uint16_t>(code);
            }
        }
        __syncthreads();
        if (threadIdx.x < 96) {
            // per axis (one warp each): the tile's count of objects in the
            // bins below each bin, an exclusive scan over the 32 bins
            const uint32_t lane = threadIdx.x & 31u, c = sb[threadIdx.x * 7];
            uint32_t inc = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t u = __shfl_up_sync(kFull, inc, off);
                if (lane >= static_cast<uint32_t>(off)) inc += u;
            }
            tile_hist[(size_t)threadIdx.x * cap_tiles + tile] = inc - c;
        }
        uint32_t* gb = bins + (size_t)ti * kBinWords;
        for (uint32_t k = threadIdx.x; k < kBinWords; k += blockDim.x) {
            const uint32_t bin = k / 7u, f = k % 7u;
            const uint32_t v = sb[k];
            if (sb[bin * 7] == 0) continue;
            if (f == 0)
                atomicAdd(gb + k, v);
            else if (f <= 3)
                atomicMin(gb + k, v);
            else
                atomicMax(gb + k, v);
        }
    }
}

// The coarse-bin window of a proposal (bucket q of 16 on an axis whose
// centroid range is [cmin, cmin + ext]): objects whose 32-bin index on that
// axis is below lo lie below every one of the proposal's thresholds
// (interval 0), above hi above every one (interval 16), and only the rest
// need their centroid compared. The 16 thresholds span
// [cmin + ext * (16q + 1) / 256, cmin + ext * (q + 1) / 16], and the coarse
// bins outside [2q - 1, 2q + 2] are at least ext / 32 away from them, far
// more than the rounding of the bin index (a few ulps of ext) and of the
// thresholds (an ulp of the coordinates), as long as the coordinates are
// within 2^14 extents of the origin; else (or without bin codes) the window
// is every bin and every object is compared, as before.
#ifndef MGBVH_REFINE_WINDOW
#define MGBVH_REFINE_WINDOW 1  // 0: the refine pass compares every object (no coarse-bin window)
#endif
#ifndef MGBVH_REFINE_BATCH
#define MGBVH_REFINE_BATCH 4  // objects a thread of the refine pass handles at a time (tuning knob; divides 8)
#endif
#ifndef MGBVH_REFINE_MIN_BLOCKS
#define MGBVH_REFINE_MIN_BLOCKS 4  // refine-pass CTAs per SM the register budget must allow (tuning knob)
#endif
constexpr uint32_t kRefineBatch = MGBVH_REFINE_BATCH;

__device__ __forceinline__ bool refine_window(float cmin, float ext, uint32_t q, uint32_t& lo, uint32_t& hi) {
    const float cmax = __fadd_rn(cmin, ext);
    const bool ok = MGBVH_REFINE_WINDOW && kPartCodes && ext > 0.0f && ext < 3.0e38f &&
                    fabsf(cmin) <= __fmul_rn(ext, 16384.0f) &&
                    fabsf(cmax) <= __fmul_rn(ext, 16384.0f);
    lo = ok && q > 0u ? 2u * q - 1u : 0u;
    hi = ok ? min(2u * q + 2u, 31u) : 31u;
    return ok;
}

// Interval bins of the pending nodes: for each proposal, the node's objects
// by the interval of their centroid among the proposal's 16 thresholds
// (count + AABB keys), with shared-memory atomics, merged into the node's
// global interval bins; per-tile running counts go to tile_hist2. Only the
// objects inside the proposal's coarse-bin window (refine_window) are read
// and compared: the bin pass's codes place the others, whose counts come
// from the tile's bin prefix counts here and whose boxes come from the
// node's coarse bins in lvl_eval2. Grid-stride over the level's tiles.
__global__ void __launch_bounds__(kTileThreads, MGBVH_REFINE_MIN_BLOCKS) lvl_refine_bin_kernel(
    const Task* __restrict__ tasks, const uint32_t* __restrict__ cbkeys,
    const LvlRefine* __restrict__ refine, uint32_t* __restrict__ rbins,
    const uint32_t* __restrict__ tile_task, const uint32_t* __restrict__ tile_begin,
    uint32_t* __restrict__ tile_hist2, const uint32_t* __restrict__ tile_hist, uint32_t cap_tiles,
    const Rec* __restrict__ rec0, const Rec* __restrict__ rec1, const uint16_t* __restrict__ codes,
    const Counters* __restrict__ ctr, uint32_t lv) {
    pdl_enter();
    __shared__ uint32_t sb[kRBinWords];
    __shared__ float sthr[32];
    const uint32_t ntiles = ctr->lvl[lv][1];
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t ti = tile_task[tile];
        const LvlRefine R = refine[ti];
        if (!R.on) continue;  // block-uniform
        __syncthreads();      // the previous tile's readers of sb are done
        for (uint32_t i = threadIdx.x; i < kRBinWords; i += blockDim.x) {
            const uint32_t f7 = i % 7u;
            sb[i] = f7 == 0 ? 0u : (f7 <= 3 ? kKeyPosInf : kKeyNegInf);
        }
        uint32_t ax[2], wlo[2], whi[2];
        bool act[2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            ax[p] = min(R.prop[p] >> 4, 2u);
            const float cmin = funkey(cbkeys[6 * ti + ax[p]]);
            const float ext = __fsub_rn(funkey(cbkeys[6 * ti + 3 + ax[p]]), cmin);
            act[p] = ext > 0.0f;
            refine_window(cmin, ext, R.prop[p] & 15u, wlo[p], whi[p]);
            if (threadIdx.x >= 16u * p && threadIdx.x < 16u * (p + 1))
                sthr[threadIdx.x] = proposal_threshold(cmin, ext, R.prop[p] & 15u, threadIdx.x & 15u);
        }
        __syncthreads();
        const Task& t = tasks[ti];
        const uint32_t begin = tile_begin[tile];
        const uint32_t cnt = min(kTile, t.len - begin);
        const Rec* src = (t.buf ? rec1 : rec0) + t.start + begin;
        const uint16_t* cs = codes + t.start + begin;
        const bool all0 = wlo[0] == 0u && whi[0] == 31u, all1 = wlo[1] == 0u && whi[1] == 31u;
        // batches of kRefineBatch objects per thread: their codes loaded
        // together, then the records of those inside a window, then compared
#pragma unroll
        for (uint32_t j0 = 0; j0 < kRecsPerThread; j0 += kRefineBatch) {
            uint32_t code[kRefineBatch];
#pragma unroll
            for (uint32_t q = 0; q < kRefineBatch; ++q) {
                const uint32_t i = threadIdx.x + (j0 + q) * kTileThreads;
                code[q] = (i < cnt && !(all0 && all1)) ? cs[i] : 0u;
            }
            bool in[kRefineBatch][2];
            float4 rl[kRefineBatch], rh[kRefineBatch];
#pragma unroll
            for (uint32_t q = 0; q < kRefineBatch; ++q) {
                const uint32_t i = threadIdx.x + (j0 + q) * kTileThreads;
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    const uint32_t b = (code[q] >> (5u * ax[p])) & 31u;
                    in[q][p] = i < cnt && act[p] && b >= wlo[p] && b <= whi[p];
                }
                if (in[q][0] || in[q][1]) {
                    rl[q] = src[i].lo;
                    rh[q] = src[i].hi;
                }
            }
#pragma unroll
            for (uint32_t q = 0; q < kRefineBatch; ++q) {
                if (!(in[q][0] || in[q][1])) continue;
                const float l[3] = {rl[q].x, rl[q].y, rl[q].z}, h[3] = {rh[q].x, rh[q].y, rh[q].z};
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    if (!in[q][p]) continue;
                    const float c = center_of(sel3(l, ax[p]), sel3(h, ax[p]));
                    // interval = number of thresholds thr with !(c < thr)
                    uint32_t lo_i = 0, hi_i = 16;
#pragma unroll
                    for (int st = 0; st < 5; ++st) {
                        if (lo_i < hi_i) {
                            const uint32_t mid = (lo_i + hi_i) >> 1;
                            if (!(c < sthr[16 * p + mid]))
                                lo_i = mid + 1;
                            else
                                hi_i = mid;
                        }
                    }
                    uint32_t* wd = sb + (p * 17 + lo_i) * 7;
                    atomicAdd(wd, 1u);
                    atomicMin(wd + 1, fkey(l[0]));
                    atomicMin(wd + 2, fkey(l[1]));
                    atomicMin(wd + 3, fkey(l[2]));
                    atomicMax(wd + 4, fkey(h[0]));
                    atomicMax(wd + 5, fkey(h[1]));
                    atomicMax(wd + 6, fkey(h[2]));
                }
            }
        }
        __syncthreads();
        if (threadIdx.x < 64) {
            // per proposal (one warp each): the tile's count of objects in
            // intervals 0..j, an inclusive scan over the 17 intervals, plus
            // the tile's objects below the window (interval 0 by their bin)
            const uint32_t lane = threadIdx.x & 31u, p = threadIdx.x >> 5;
            const uint32_t c = lane < 17 ? sb[(p * 17 + lane) * 7] : 0u;
            uint32_t inc = c;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t u = __shfl_up_sync(kFull, inc, off);
                if (lane >= static_cast<uint32_t>(off)) inc += u;
            }
            const uint32_t below = wlo[p] ? tile_hist[(size_t)(ax[p] * 32u + wlo[p]) * cap_tiles + tile] : 0u;
            if (lane < 16) tile_hist2[(size_t)(p * 17 + lane) * cap_tiles + tile] = inc + below;
            if (lane == 16) tile_hist2[(size_t)(p * 17 + 16) * cap_tiles + tile] = cnt;
        }
        uint32_t* gb = rbins + (size_t)ti * kRBinWords;
        for (uint32_t k = threadIdx.x; k < kRBinWords; k += blockDim.x) {
            const uint32_t r = k / 7u, f7 = k % 7u;
            if (sb[r * 7] == 0) continue;
            if (f7 == 0)
                atomicAdd(gb + k, sb[k]);
            else if (f7 <= 3)
                atomicMin(gb + k, sb[k]);
            else
                atomicMax(gb + k, sb[k]);
        }
    }
}

// Pending nodes: lane p * 16 + k scores threshold k of proposal p exactly
// from the interval bins (lt = intervals 0..k, gt = k + 1..16); the first
// minimum of (cost, axis, lane) replaces the binned split when strictly
// cheaper; then the node and its children are written.
__device__ void eval2_task(const EvalArgs& A, const Params& P, const Out& O, uint32_t w, uint32_t lane) {
    const Task t = A.tasks[w];
    Decision d = A.dec[w];
    const LvlRefine R = A.refine[w];
    const uint32_t p = lane >> 4, k = lane & 15u;
    const uint32_t a = min(R.prop[p] >> 4, 2u);
    const float cmin = funkey(A.cbkeys[6 * w + a]);
    const float ext = __fsub_rn(funkey(A.cbkeys[6 * w + 3 + a]), cmin);
    const float thr = proposal_threshold(cmin, ext, R.prop[p] & 15u, k);
    const uint32_t* rb = A.rbins + (size_t)w * kRBinWords + p * 17u * 7u;
    float lt[6], gt[6];
    box_empty(lt);
    box_empty(gt);
    uint32_t nl = 0, ng = 0;
    // the objects outside the proposal's coarse-bin window: the node's coarse
    // bins below it (interval 0) and above it (interval 16), merged across
    // the proposal's 16 lanes (lane k takes bins k and k + 16)
    uint32_t win_lo = 0, win_hi = 31;
    refine_window(cmin, ext, R.prop[p] & 15u, win_lo, win_hi);
    uint32_t e0 = 0, e16 = 0;
    uint32_t k0[6] = {kKeyPosInf, kKeyPosInf, kKeyPosInf, kKeyNegInf, kKeyNegInf, kKeyNegInf};
    uint32_t k16[6] = {kKeyPosInf, kKeyPosInf, kKeyPosInf, kKeyNegInf, kKeyNegInf, kKeyNegInf};
    const uint32_t* cbn = A.bins + (size_t)w * kBinWords + a * 32u * 7u;
#pragma unroll
    for (uint32_t h = 0; h < 2; ++h) {
        const uint32_t bin = k + 16u * h;
        const bool lo_side = bin < win_lo, hi_side = bin > win_hi;
        if (!(lo_side || hi_side)) continue;
        const uint32_t* bw = cbn + bin * 7u;
        const uint32_t c = bw[0];
        if (c == 0) continue;
        if (lo_side)
            e0 += c;
        else
            e16 += c;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const uint32_t v = bw[1 + i];
            if (lo_side)
                k0[i] = i < 3 ? min(k0[i], v) : max(k0[i], v);
            else
                k16[i] = i < 3 ? min(k16[i], v) : max(k16[i], v);
        }
    }
#pragma unroll
    for (int off = 8; off > 0; off >>= 1) {  // within the proposal's 16 lanes
        e0 += __shfl_xor_sync(kFull, e0, off);
        e16 += __shfl_xor_sync(kFull, e16, off);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const uint32_t u0 = __shfl_xor_sync(kFull, k0[i], off), u16 = __shfl_xor_sync(kFull, k16[i], off);
            k0[i] = i < 3 ? min(k0[i], u0) : max(k0[i], u0);
            k16[i] = i < 3 ? min(k16[i], u16) : max(k16[i], u16);
        }
    }
    uint32_t cj[17];
#pragma unroll
    for (uint32_t j = 0; j < 17; ++j) cj[j] = rb[j * 7];  // all counts in flight at once
#pragma unroll
    for (uint32_t j = 0; j < 17; ++j) {
        const uint32_t* b = rb + j * 7;
        const uint32_t c = cj[j];
        if (c == 0) continue;
        if (j <= k)
            nl += c;
        else
            ng += c;
        box_grow2(lt, gt, j <= k, funkey(b[1]), funkey(b[2]), funkey(b[3]), funkey(b[4]), funkey(b[5]),
                  funkey(b[6]));
    }
    if (e0) {  // interval 0 is on the lt side of every threshold
        nl += e0;
        box_grow2(lt, gt, true, funkey(k0[0]), funkey(k0[1]), funkey(k0[2]), funkey(k0[3]), funkey(k0[4]),
                  funkey(k0[5]));
    }
    if (e16) {  // interval 16 is on the gt side of every threshold
        ng += e16;
        box_grow2(lt, gt, false, funkey(k16[0]), funkey(k16[1]), funkey(k16[2]), funkey(k16[3]),
                  funkey(k16[4]), funkey(k16[5]));
    }
    const float nb[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
    uint64_t key = ~0ull;
    if (ext > 0.0f && nl >= P.min_leaf && ng >= P.min_leaf)
        key = cand_key(split_cost(surface_area6(lt), surface_area6(gt), surface_area6(nb), nl, ng), a, lane);
    const uint64_t wk = warp_min_key(key);
    const uint32_t wlo = static_cast<uint32_t>(wk);
    if (wlo != kNoKey && static_cast<uint32_t>(wk >> 32) < d.plain_key) {
        const uint32_t src = wlo & 0xFFu;
        d.use_thr = 1;
        d.axis = (wlo >> 8) & 3u;
        d.thr = __shfl_sync(kFull, thr, src);
        d.n_lt = __shfl_sync(kFull, nl, src);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            d.ltb[i] = __shfl_sync(kFull, lt[i], src);
            d.gtb[i] = __shfl_sync(kFull, gt[i], src);
        }
        if (lane == 0) atomicAdd(&O.ctr->learned, 1u);
        emit_split(A, P, O, w, lane, t, d, A.tile_hist2, (src >> 4) * 17u + (src & 15u));
    } else {
        emit_split(A, P, O, w, lane, t, d, A.tile_hist, d.axis * 32u + d.split_bin);
    }
}

__global__ void __launch_bounds__(128) lvl_eval2_kernel(EvalArgs A, Params P, Out O) {
    pdl_enter();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n_tasks = O.ctr->lvl[A.lv][0];
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_tasks; w += nwarps)
        if (A.refine[w].on) eval2_task(A, P, O, w, lane);
}

// Training samples of the level-pass nodes of at most kSampleLargeMax
// objects that took a binned split: one CTA per node computes the exact
// full sweep (every centroid a threshold on every axis; first minimum of
// (cost, axis, threshold)), one thread per threshold, the node's records
// streamed through shared memory; warp 0 then writes the sample.
constexpr uint32_t kSampleChunk = 1024;

__global__ void __launch_bounds__(256) lvl_sample_kernel(const Task* __restrict__ tasks,
                                                         const Decision* __restrict__ dec,
                                                         const uint32_t* __restrict__ bins,
                                                         const uint32_t* __restrict__ cbkeys,
                                                         const Rec* __restrict__ rec0,
                                                         const Rec* __restrict__ rec1,
                                                         const Counters* __restrict__ ctr, uint32_t lv,
                                                         Params P, Learn LN) {
    pdl_enter();
    __shared__ float3 slo[kSampleChunk], shi[kSampleChunk];
    __shared__ uint32_t rk[8], ra[8], rt[8];
    __shared__ float rthr[8];
    const uint32_t n_tasks = ctr->lvl[lv][0];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if ((P.bins ? P.bins : 32u) != 32u) return;
    for (uint32_t w = blockIdx.x; w < n_tasks; w += gridDim.x) {
        const Task t = tasks[w];
        const Decision d = dec[w];
        if (d.kind != 0 || t.len > kSampleLargeMax) continue;  // block-uniform
        const uint32_t n = t.len;
        const Rec* src = (t.buf ? rec1 : rec0) + t.start;
        const float nb[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
        const float sa_p = surface_area6(nb);
        uint32_t bk = kNoKey, ba = 3, bt = kNoKey;
        float bthr = 0.0f;
        for (uint32_t a = 0; a < 3; ++a) {
            for (uint32_t k0 = 0; k0 < n; k0 += blockDim.x) {
                const uint32_t kk = k0 + threadIdx.x;
                float thr = 0.0f;
                if (kk < n) {
                    const float* lo = reinterpret_cast<const float*>(&src[kk].lo);
                    const float* hi = reinterpret_cast<const float*>(&src[kk].hi);
                    thr = center_of(lo[a], hi[a]);
                }
                float blt[6], bgt[6];
                box_empty(blt);
                box_empty(bgt);
                uint32_t nl = 0;
                for (uint32_t c0 = 0; c0 < n; c0 += kSampleChunk) {
                    const uint32_t m = min(kSampleChunk, n - c0);
                    __syncthreads();
                    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                        const Rec r = src[c0 + i];
                        slo[i] = make_float3(r.lo.x, r.lo.y, r.lo.z);
                        shi[i] = make_float3(r.hi.x, r.hi.y, r.hi.z);
                    }
                    __syncthreads();
                    for (uint32_t j = 0; j < m; ++j) {
                        const float3 l = slo[j], h = shi[j];
                        const float cj = center_of(a == 0 ? l.x : (a == 1 ? l.y : l.z),
                                                   a == 0 ? h.x : (a == 1 ? h.y : h.z));
                        if (cj < thr) {
                            box_grow(blt, l.x, l.y, l.z, h.x, h.y, h.z);
                            nl++;
                        } else {
                            box_grow(bgt, l.x, l.y, l.z, h.x, h.y, h.z);
                        }
                    }
                }
                const uint32_t ng = n - nl;
                if (kk < n && nl >= P.min_leaf && ng >= P.min_leaf) {
                    const uint32_t ck = fkey(split_cost(surface_area6(blt), surface_area6(bgt), sa_p, nl, ng));
                    const uint32_t tk = fkey(thr);
                    if (ck < bk || (ck == bk && (a < ba || (a == ba && tk < bt)))) {
                        bk = ck;
                        ba = a;
                        bt = tk;
                        bthr = thr;
                    }
                }
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const uint32_t ok = __shfl_xor_sync(kFull, bk, off);
            const uint32_t oa = __shfl_xor_sync(kFull, ba, off);
            const uint32_t ot = __shfl_xor_sync(kFull, bt, off);
            const float oth = __shfl_xor_sync(kFull, bthr, off);
            if (ok < bk || (ok == bk && (oa < ba || (oa == ba && ot < bt)))) {
                bk = ok;
                ba = oa;
                bt = ot;
                bthr = oth;
            }
        }
        if (lane == 0) {
            rk[warp] = bk;
            ra[warp] = ba;
            rt[warp] = bt;
            rthr[warp] = bthr;
        }
        __syncthreads();
        if (warp == 0) {
            bk = lane < 8 ? rk[lane] : kNoKey;
            ba = lane < 8 ? ra[lane] : 3u;
            bt = lane < 8 ? rt[lane] : kNoKey;
            bthr = lane < 8 ? rthr[lane] : 0.0f;
            for (int off = 16; off > 0; off >>= 1) {
                const uint32_t ok = __shfl_xor_sync(kFull, bk, off);
                const uint32_t oa = __shfl_xor_sync(kFull, ba, off);
                const uint32_t ot = __shfl_xor_sync(kFull, bt, off);
                const float oth = __shfl_xor_sync(kFull, bthr, off);
                if (ok < bk || (ok == bk && (oa < ba || (oa == ba && ot < bt)))) {
                    bk = ok;
                    ba = oa;
                    bt = ot;
                    bthr = oth;
                }
            }
            float cb[6];
            for (int a = 0; a < 6; ++a) cb[a] = funkey(cbkeys[6 * w + a]);
            uint32_t cnt[3];
            for (int a = 0; a < 3; ++a)
                cnt[a] = cb[3 + a] - cb[a] == 0.0f ? 0u : bins[(size_t)w * kBinWords + (a * 32 + lane) * 7];
            float f[24];
            node_features(nb, cb, n, t.depth, cnt, f);
            if (lane == 0) {
                const float cmin_a = ba < 3 ? cb[ba] : 0.0f;
                const float ext_a = ba < 3 ? __fsub_rn(cb[3 + ba], cb[ba]) : 0.0f;
                write_sample(LN, f, bk, ba, bthr, cmin_a, ext_a, d.plain_key, n, t.start - t.tbase);
            }
        }
    }
}

// Stable partition of the large nodes' records into the other buffer: lt
// records to the front of the node in order, gt records after them in order.
// Each warp owns 256 consecutive records of the tile: a first pass computes
// the side of each record (kept as 8 ballot words), one barrier publishes the
// per-warp lt counts, and a second pass re-reads the records (cache hits) and
// scatters them. Grid-stride over the level's tiles; also reduces the large
// children's centroid bounds.
constexpr uint32_t kPartPerLane = kTile / kTileThreads;  // 8

#ifndef MGBVH_PART_MIN_BLOCKS
#define MGBVH_PART_MIN_BLOCKS 5  // CTAs per SM the register budget must allow (tuning knob)
#endif

__global__ void __launch_bounds__(kTileThreads, MGBVH_PART_MIN_BLOCKS) lvl_part_kernel(
    const Task* __restrict__ tasks, const Decision* __restrict__ dec,
    const uint32_t* __restrict__ tile_task, const uint32_t* __restrict__ tile_begin,
    const uint32_t* __restrict__ tile_lt, Rec* rec0, Rec* rec1, const uint16_t* __restrict__ codes,
    uint32_t* next_cbkeys, uint32_t lv, Out O) {
    pdl_enter();
    __shared__ uint32_t wcnt[kTileThreads / 32];
    __shared__ uint32_t sk[12];
    __shared__ int sbad;
    const uint32_t ntiles = O.ctr->lvl[lv][1];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t below = (1u << lane) - 1u;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t ti = tile_task[tile];
        const Task& t = tasks[ti];
        const Decision& d = dec[ti];
        const uint32_t begin = tile_begin[tile];
        const uint32_t tstart = t.start, tlen = t.len;
        const uint32_t cnt = min(kTile, tlen - begin);
        const Rec* src = (t.buf ? rec1 : rec0) + tstart + begin;
        Rec* dst = t.buf ? rec0 : rec1;
        if (d.kind == 1) {
            for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x)
                O.perm[tstart + begin + i] = __float_as_uint(src[i].lo.w);
            continue;
        }
        const uint32_t axis = d.axis, split_bin = d.split_bin, nbins = d.bins, n_lt = d.n_lt;
        const float cmin = d.cmin, ext = d.ext, thr = d.thr;
        const bool use_thr = d.use_thr != 0;
        if (threadIdx.x < 12) sk[threadIdx.x] = ((threadIdx.x % 6) < 3) ? kKeyPosInf : kKeyNegInf;
        if (threadIdx.x == 0) sbad = 0;
        const uint32_t w0 = warp * (32u * kPartPerLane);
        // pass 1: sides (from the bin pass's codes for a binned split; else the
        // split axis's bounds of all this lane's records are loaded first)
        uint32_t bal[kPartPerLane];
        uint32_t lt_w = 0;
        if (kPartCodes && !use_thr) {
            // binned split: the bin pass left each record's bin on the split axis
            const uint16_t* cs = codes + tstart + begin;
            const uint32_t sh = 5u * axis;
            uint32_t cj[kPartPerLane];
#pragma unroll
            for (uint32_t j = 0; j < kPartPerLane; ++j) {
                const uint32_t i = w0 + j * 32u + lane;
                cj[j] = i < cnt ? cs[i] : 0xFFFFu;
            }
#pragma unroll
            for (uint32_t j = 0; j < kPartPerLane; ++j) {
                const bool pred = w0 + j * 32u + lane < cnt && ((cj[j] >> sh) & 31u) < split_bin;
                bal[j] = __ballot_sync(kFull, pred);
                lt_w += __popc(bal[j]);
            }
        } else {
            float pl[kPartPerLane], ph[kPartPerLane];
#pragma unroll
            for (uint32_t j = 0; j < kPartPerLane; ++j) {
                const uint32_t i = w0 + j * 32u + lane;
                if (i < cnt) {
                    pl[j] = reinterpret_cast<const float*>(&src[i].lo)[axis];
                    ph[j] = reinterpret_cast<const float*>(&src[i].hi)[axis];
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < kPartPerLane; ++j) {
                const uint32_t i = w0 + j * 32u + lane;
                bool pred = false;
                if (i < cnt) {
                    const float c = center_of(pl[j], ph[j]);
                    pred = use_thr ? c < thr : bin_of(c, cmin, ext, nbins) < split_bin;
                }
                bal[j] = __ballot_sync(kFull, pred);
                lt_w += __popc(bal[j]);
            }
        }
        if (lane == 0) wcnt[warp] = lt_w;
        __syncthreads();
        uint32_t run = 0;
        for (uint32_t q = 0; q < warp; ++q) run += wcnt[q];
        const uint32_t lt_off = tile_lt[tile];
        const uint32_t lt_base = tstart + lt_off;
        const uint32_t gt_base = tstart + n_lt + (begin - lt_off);
        const bool leaf_lt = d.child_leaf[1] != 0, leaf_gt = d.child_leaf[0] != 0;
        uint32_t k[12];
        init_key12(k);
        bool bad = false;
        // pass 2: scatter
#pragma unroll(kPartUnroll)
        for (uint32_t j = 0; j < kPartPerLane; ++j) {
            const uint32_t i = w0 + j * 32u + lane;
            if (i < cnt) {
                const Rec r = src[i];
                const bool pred = (bal[j] >> lane) & 1u;
                const uint32_t ltr = run + __popc(bal[j] & below);
                const uint32_t dest = pred ? lt_base + ltr : gt_base + (i - ltr);
                const float c0 = center_of(r.lo.x, r.hi.x), c1 = center_of(r.lo.y, r.hi.y),
                            c2 = center_of(r.lo.z, r.hi.z);
                if (dest - tstart < tlen) {
                    dst[dest] = r;
                    if (pred ? leaf_lt : leaf_gt) O.perm[dest] = __float_as_uint(r.lo.w);
                } else {
                    bad = true;  // inconsistent counts; never write outside the node
                }
                bad |= !box_contains(pred ? d.ltb : d.gtb, c0, c1, c2);
                const float c[3] = {c0, c1, c2};
                grow_keys12(k, pred, c);
            }
            run += __popc(bal[j]);
        }
        const bool need_lt = d.child_task[1] != kNone, need_gt = d.child_task[0] != kNone;
        if (need_lt || need_gt) {
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                const bool is_min = (q % 6) < 3;
                const uint32_t v = is_min ? __reduce_min_sync(kFull, k[q]) : __reduce_max_sync(kFull, k[q]);
                if (lane == 0) {
                    if (is_min)
                        atomicMin(&sk[q], v);
                    else
                        atomicMax(&sk[q], v);
                }
            }
        }
        if (__any_sync(kFull, bad) && lane == 0) sbad = 1;
        __syncthreads();
        if (threadIdx.x == 0 && sbad) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteContain);
        if ((need_lt || need_gt) && threadIdx.x < 12) {
            const uint32_t q = threadIdx.x;
            const uint32_t child = q < 6 ? d.child_task[1] : d.child_task[0];
            if (child != kNone) {
                uint32_t* g = next_cbkeys + 6 * child + (q % 6);
                if ((q % 6) < 3)
                    atomicMin(g, sk[q]);
                else
                    atomicMax(g, sk[q]);
            }
        }
        __syncthreads();  // wcnt/sk/sbad are rewritten by the next tile
    }
}

// ---------------------------------------------------------------- forced median of large nodes
//
// median_split (bvh/src/lib.rs:444-491) on axes 0, 1 and 2 in turn over the
// same list (:527-531), for the level-pass nodes whose binned sweeps all
// refused (lvl_eval_kernel queues them). The waiting nodes' objects form one
// element range, node s owning elements moff[s] .. moff[s+1] in list order.
// Per axis:
//   med_key_kernel      (node, centroid key) per element, position as value
//   radix sort          stable, so equal keys stay in list order
//   med_flag_kernel     element in lt <=> (key, position) <= the node's m-th
//                       smallest pair, m = len / 2: the set
//                       select_nth_unstable_by(m, total_cmp) puts first, ties
//                       taken in list order
//   exclusive scan      of the flags
//   med_scatter_kernel  stable partition into the other record buffer; box
//                       keys of both halves on this axis
// Axis 0 moves the records buf -> buf^1, axis 1 back, axis 2 to buf^1 (the
// children's buffer): the list ends in axis-2 order whichever axis wins, as
// in the reference. med_finish_kernel takes the cheapest axis (first minimum
// of total_cmp), applies the containment assertion (:637-646) to the final
// halves and writes the node and its children.

struct MedSeg {
    uint32_t box[3][12];  // per axis: lt box keys (lo xyz, hi xyz), then gt box keys
    uint32_t ckeys[12];   // centroid keys of the final halves: lt lo xyz, lt hi xyz, gt lo xyz, gt hi xyz
};

// Where a median node's children go (the next pipeline run starts at level 0).
struct MedOut {
    Task* tasks;
    uint32_t* bins;
    uint32_t* cbkeys;
    uint32_t* tile_task;
    uint32_t* tile_begin;
    Task* medium;
    Task* small;
    uint32_t cap_tasks, cap_tiles, cap_medium, cap_small;
};

__device__ __forceinline__ bool child_is_leaf(uint32_t len, uint32_t depth, const Params& P) {
    return len <= 1u || depth == P.max_depth || (len <= P.max_leaf && len < 2u * P.min_leaf);
}

// The waiting node that owns element e: the last s with moff[s] <= e.
__device__ __forceinline__ uint32_t med_node_of(const uint32_t* __restrict__ moff, uint32_t np, uint32_t e) {
    uint32_t lo = 0, hi = np;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (moff[mid] <= e)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void med_reset_kernel(Counters* ctr) {
    if (threadIdx.x < 6) ctr->lvl[threadIdx.x >> 1][threadIdx.x & 1u] = 0;
    if (threadIdx.x == 0) {
        ctr->n_medium = 0;
        ctr->n_small = 0;
        ctr->n_med = 0;
        ctr->medium_take = 0;
        ctr->small_take = 0;
    }
}

__global__ void med_init_kernel(MedSeg* seg, uint32_t np) {
    const uint32_t words = sizeof(MedSeg) / 4;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np * words; i += gridDim.x * blockDim.x) {
        const uint32_t q = (i % words) % 6u;
        reinterpret_cast<uint32_t*>(seg)[i] = q < 3 ? kKeyPosInf : kKeyNegInf;
    }
}

__global__ void __launch_bounds__(256) med_key_kernel(const Task* __restrict__ mt, const uint32_t* __restrict__ moff,
                                                      uint32_t np, uint32_t E, const Rec* __restrict__ rec0,
                                                      const Rec* __restrict__ rec1, uint32_t axis,
                                                      unsigned long long* __restrict__ keys,
                                                      uint32_t* __restrict__ vals) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        const uint32_t s = med_node_of(moff, np, e);
        const uint32_t i = e - moff[s];
        const Rec* src = ((mt[s].buf ^ (axis & 1u)) ? rec1 : rec0) + mt[s].start;
        const float lo = reinterpret_cast<const float*>(&src[i].lo)[axis];
        const float hi = reinterpret_cast<const float*>(&src[i].hi)[axis];
        keys[e] = (static_cast<unsigned long long>(s) << 32) | fkey(center_of(lo, hi));
        vals[e] = i;
    }
}

__global__ void __launch_bounds__(256) med_flag_kernel(const Task* __restrict__ mt, const uint32_t* __restrict__ moff,
                                                       uint32_t np, uint32_t E,
                                                       const unsigned long long* __restrict__ keys,
                                                       const unsigned long long* __restrict__ sorted_keys,
                                                       const uint32_t* __restrict__ sorted_vals,
                                                       uint32_t* __restrict__ flag) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        const uint32_t s = med_node_of(moff, np, e);
        const uint32_t i = e - moff[s];
        const uint32_t c = moff[s] + mt[s].len / 2u - 1u;  // the m-th smallest (key, position)
        const uint32_t cut_key = static_cast<uint32_t>(sorted_keys[c]), cut_pos = sorted_vals[c];
        const uint32_t k = static_cast<uint32_t>(keys[e]);
        flag[e] = (k < cut_key || (k == cut_key && i <= cut_pos)) ? 1u : 0u;
    }
}

__global__ void __launch_bounds__(256) med_scatter_kernel(const Task* __restrict__ mt,
                                                          const uint32_t* __restrict__ moff, uint32_t np,
                                                          uint32_t E, Rec* rec0, Rec* rec1, uint32_t axis,
                                                          const uint32_t* __restrict__ flag,
                                                          const uint32_t* __restrict__ scan, MedSeg* seg,
                                                          Params P, Out O) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    // whole warps step together (the reductions below take every lane)
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < E; base += nwarps * 32u) {
        const uint32_t e = base + lane;
        const bool valid = e < E;
        uint32_t s = 0, bk[6], ck[3];
        bool lt = false;
        if (valid) {
            s = med_node_of(moff, np, e);
            const Task& t = mt[s];
            const uint32_t i = e - moff[s], m = t.len / 2u;
            const uint32_t sb = t.buf ^ (axis & 1u);
            const Rec r = ((sb ? rec1 : rec0) + t.start)[i];
            lt = flag[e] != 0u;
            const uint32_t lt_before = scan[e] - scan[moff[s]];
            const uint32_t pos = lt ? lt_before : m + (i - lt_before);
            if (pos < t.len) {
                ((sb ? rec0 : rec1) + t.start)[pos] = r;
                // axis 2 leaves the final order: a leaf child's objects are placed
                if (axis == 2u && child_is_leaf(lt ? m : t.len - m, t.depth + 1u, P))
                    O.perm[t.start + pos] = __float_as_uint(r.lo.w);
            } else {
                set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteMedian);
            }
            bk[0] = fkey(r.lo.x);
            bk[1] = fkey(r.lo.y);
            bk[2] = fkey(r.lo.z);
            bk[3] = fkey(r.hi.x);
            bk[4] = fkey(r.hi.y);
            bk[5] = fkey(r.hi.z);
            ck[0] = fkey(center_of(r.lo.x, r.hi.x));
            ck[1] = fkey(center_of(r.lo.y, r.hi.y));
            ck[2] = fkey(center_of(r.lo.z, r.hi.z));
        }
        const uint32_t s0 = __shfl_sync(kFull, s, 0);
        if (__all_sync(kFull, !valid || s == s0)) {
            // one node under the whole warp: reduce per half, then one atomic per word
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                const bool mine = valid && (lt == (q < 6));
                const bool is_min = (q % 6) < 3;
                const uint32_t v = mine ? bk[q % 6] : (is_min ? kKeyPosInf : kKeyNegInf);
                const uint32_t r = is_min ? __reduce_min_sync(kFull, v) : __reduce_max_sync(kFull, v);
                if (lane == 0) {
                    if (is_min)
                        atomicMin(&seg[s0].box[axis][q], r);
                    else
                        atomicMax(&seg[s0].box[axis][q], r);
                }
            }
            if (axis == 2u) {
#pragma unroll
                for (int q = 0; q < 12; ++q) {
                    const bool mine = valid && (lt == (q < 6));
                    const bool is_min = (q % 6) < 3;
                    const uint32_t v = mine ? ck[q % 3] : (is_min ? kKeyPosInf : kKeyNegInf);
                    const uint32_t r = is_min ? __reduce_min_sync(kFull, v) : __reduce_max_sync(kFull, v);
                    if (lane == 0) {
                        if (is_min)
                            atomicMin(&seg[s0].ckeys[q], r);
                        else
                            atomicMax(&seg[s0].ckeys[q], r);
                    }
                }
            }
        } else if (valid) {
            // a node boundary inside the warp: per-lane atomics
            uint32_t* b = seg[s].box[axis] + (lt ? 0 : 6);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                atomicMin(b + q, bk[q]);
                atomicMax(b + 3 + q, bk[3 + q]);
            }
            if (axis == 2u) {
                uint32_t* c = seg[s].ckeys + (lt ? 0 : 6);
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    atomicMin(c + q, ck[q]);
                    atomicMax(c + 3 + q, ck[q]);
                }
            }
        }
    }
}

// One warp per median node: the cheapest axis, the containment assertion,
// the node and its two children (leaf, level-pass task, subtree CTA task or
// warp subtree task).
__global__ void __launch_bounds__(128) med_finish_kernel(const Task* __restrict__ mt, uint32_t np,
                                                         const MedSeg* __restrict__ seg, MedOut M, Params P,
                                                         Out O) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < np; s += nwarps) {
        const Task t = mt[s];
        const MedSeg& G = seg[s];
        const uint32_t n = t.len, m = n / 2u;
        const float nb[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
        uint64_t key = ~0ull;
        if (lane < 3) {
            float lb[6], gb[6];
            for (int q = 0; q < 6; ++q) {
                lb[q] = funkey(G.box[lane][q]);
                gb[q] = funkey(G.box[lane][6 + q]);
            }
            key = cand_key(split_cost(surface_area6(lb), surface_area6(gb), surface_area6(nb), m, n - m), lane, 0u);
        }
        const uint32_t axis = (static_cast<uint32_t>(warp_min_key(key)) >> 8) & 3u;
        float ltb[6], gtb[6];
        for (int q = 0; q < 6; ++q) {
            ltb[q] = funkey(G.box[axis][q]);
            gtb[q] = funkey(G.box[axis][6 + q]);
        }
        // every centroid of a half inside that half's box: the corners of the
        // half's centroid bounds inside it
        const uint32_t* ck = G.ckeys;
        const bool ok = box_contains(ltb, funkey(ck[0]), funkey(ck[1]), funkey(ck[2])) &&
                        box_contains(ltb, funkey(ck[3]), funkey(ck[4]), funkey(ck[5])) &&
                        box_contains(gtb, funkey(ck[6]), funkey(ck[7]), funkey(ck[8])) &&
                        box_contains(gtb, funkey(ck[9]), funkey(ck[10]), funkey(ck[11]));
        if (!ok) {
            if (lane == 0) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteContain);
            continue;
        }
        warp_store_node(O, t.nbase + t.slot, nb, t.start - t.tbase, n, t.pair, lane);
        if (lane == 0) {
            atomicMax(&O.ctr->height, t.depth);
            atomicAdd(&O.ctr->median_splits, 1u);
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {  // [0] gt, [1] lt, as the reference pushes them
            const uint32_t len = c == 0 ? n - m : m;
            const uint32_t start = c == 0 ? t.start + m : t.start;
            const uint32_t slot = c == 0 ? t.pair : t.pair + 1u;
            const uint32_t depth = t.depth + 1u;
            float cb[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) cb[q] = c == 0 ? gtb[q] : ltb[q];
            if (child_is_leaf(len, depth, P)) {
                warp_store_node(O, t.nbase + slot, cb, start - t.tbase, len, 0u, lane);
                if (lane == 0 && len > 1) {
                    atomicAdd(&O.ctr->holes, 1u);
                    if (depth == P.max_depth) atomicAdd(&O.ctr->depth_capped, 1u);
                }
                continue;
            }
            Task ct;
            for (int a = 0; a < 3; ++a) {
                ct.lo[a] = cb[a];
                ct.hi[a] = cb[3 + a];
            }
            ct.start = start;
            ct.len = len;
            ct.slot = slot;
            ct.pair = c == 0 ? t.pair + 2u : t.pair + 2u * (n - m);
            ct.depth = depth;
            ct.buf = t.buf ^ 1u;
            ct.tile0 = ct.ntiles = 0;
            ct.nbase = t.nbase;
            ct.tbase = t.tbase;
            if (len > P.medium_max) {
                const uint32_t nt = (len + kTile - 1) / kTile;
                uint32_t ti = 0, t0 = 0;
                if (lane == 0) {
                    ti = atomicAdd(&O.ctr->lvl[0][0], 1u);
                    t0 = atomicAdd(&O.ctr->lvl[0][1], nt);
                }
                ti = __shfl_sync(kFull, ti, 0);
                t0 = __shfl_sync(kFull, t0, 0);
                if (ti >= M.cap_tasks || t0 + nt > M.cap_tiles) {
                    if (lane == 0) set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                    continue;
                }
                ct.tile0 = t0;
                ct.ntiles = nt;
                if (lane == 0) M.tasks[ti] = ct;
                init_task_bins(M.bins + (size_t)ti * kBinWords, lane, 32);
                if (lane < 6) M.cbkeys[6 * ti + lane] = ck[(c == 0 ? 6 : 0) + lane];
                for (uint32_t i = lane; i < nt; i += 32) {
                    M.tile_task[t0 + i] = ti;
                    M.tile_begin[t0 + i] = i * kTile;
                }
            } else {
                const bool med = len > kSmallMax;
                uint32_t li = 0;
                if (lane == 0) li = atomicAdd(med ? &O.ctr->n_medium : &O.ctr->n_small, 1u);
                li = __shfl_sync(kFull, li, 0);
                if (li >= (med ? M.cap_medium : M.cap_small)) {
                    if (lane == 0) set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                    continue;
                }
                if (lane == 0) (med ? M.medium : M.small)[li] = ct;
            }
        }
    }
}

// ---------------------------------------------------------------- medium

struct MNode {  // 64 bytes
    float b[6];
    float cb[6];
    uint32_t s, n, slot, pair;
};
struct MNodeExtra {
    uint32_t depth, ib;
};

// Shared memory of one subtree CTA for subtrees of up to kCap objects: the
// records, two index lists, two node lists (every listed node holds more than
// 32 objects and the nodes of one list are disjoint, so kCap / 33 + 1 entries
// suffice), per-warp bins and exchange space.
template <uint32_t kCap>
struct MediumSmemT {
    static constexpr uint32_t kListCap = kCap / (kSmallMax + 1) + 1;
    float4 rlo[kCap];
    float4 rhi[kCap];
    uint16_t idx[2][kCap];
    MNode list[2][kListCap];
    MNodeExtra list_x[2][kListCap];
    uint32_t bins[kMediumWarps][kBinWords];
    XRec xchg[kMediumWarps][32];
    uint32_t list_n[2];
    uint32_t rootk[12];
};
using MediumSmem = MediumSmemT<kMediumMax>;
constexpr uint32_t kMediumSmallCap = 512;  // the instance for medium_max <= 512 (more CTAs per SM)
using MediumSmemSmall = MediumSmemT<kMediumSmallCap>;

// A subtree of <= 32 objects split off inside a subtree CTA of the persistent
// build: its objects are idx[ob][cs .. cs + len) of the CTA's records, built
// by the CTA's warps once the CTA's own nodes are done (the range is the
// subtree's alone, so later partitions leave it as it is).
struct SmallRef {
    float b[6];
    uint32_t slot, pair, depth;
    uint16_t cs;
    uint8_t len, ob;
};

// The persistent build's subtree CTA: the records, lists and bins of a
// subtree CTA, plus the list of its subtrees of <= 32 objects (at most
// kCap / 2: disjoint subtrees of at least 2 objects).
template <uint32_t kCap>
struct MediumSmemQ : MediumSmemT<kCap> {
    SmallRef sref[kCap / 2];
    uint32_t sref_n;
};

template <class MS>
__device__ __forceinline__ void medium_load_warp_records(const MS& S, uint32_t ib, uint32_t s,
                                                         uint32_t n, uint32_t lane, float* lo,
                                                         float* hi, uint32_t& id) {
    if (lane < n) {
        const uint32_t r = S.idx[ib][s + lane];
        const float4 a = S.rlo[r], b = S.rhi[r];
        lo[0] = a.x;
        lo[1] = a.y;
        lo[2] = a.z;
        id = __float_as_uint(a.w);
        hi[0] = b.x;
        hi[1] = b.y;
        hi[2] = b.z;
    } else {
        lo[0] = lo[1] = lo[2] = hi[0] = hi[1] = hi[2] = 0.0f;
        id = 0;
    }
}

// Warp: finish a leaf of the medium subtree (record + permutation).
template <class MS>
__device__ __forceinline__ void medium_leaf(const MS& S, uint32_t ib, uint32_t base,
                                            uint32_t s, uint32_t n, uint32_t slot, uint32_t depth,
                                            const float* b, uint32_t nbase, uint32_t tbase,
                                            const Params& P, const Out& O, uint32_t lane) {
    warp_store_node(O, nbase + slot, b, base + s - tbase, n, 0u, lane);
    for (uint32_t p = lane; p < n; p += 32)
        O.perm[base + s + p] = __float_as_uint(S.rlo[S.idx[ib][s + p]].w);
    if (lane == 0 && n > 1) {
        atomicAdd(&O.ctr->holes, 1u);
        if (depth == P.max_depth) atomicAdd(&O.ctr->depth_capped, 1u);
    }
}

// Warp: stable partition of [s, s+n) from idx[ib] into idx[ib^1] by pred(p);
// returns the lt count; accumulates child centroid keys.
// With clt non-null, also checks each centroid against its side's child box
// (clt for lt, cgt for gt) and sets bad where one lies outside.
template <class MS, class Pred>
__device__ __forceinline__ uint32_t medium_partition(MS& S, uint32_t ib, uint32_t s,
                                                     uint32_t n, uint32_t n_lt_expect, uint32_t lane,
                                                     Pred pred, uint32_t* k /*12*/,
                                                     const float* clt = nullptr,
                                                     const float* cgt = nullptr, bool* bad = nullptr) {
    const uint32_t below = (1u << lane) - 1u;
    uint32_t lt_run = 0, gt_run = 0;
    for (uint32_t b0 = s; b0 < s + n; b0 += 32) {
        const uint32_t p = b0 + lane;
        const bool valid = p < s + n;
        uint32_t r = 0;
        float c[3] = {0.f, 0.f, 0.f};
        bool pr = false;
        if (valid) {
            r = S.idx[ib][p];
            const float4 a = S.rlo[r], b = S.rhi[r];
            c[0] = center_of(a.x, b.x);
            c[1] = center_of(a.y, b.y);
            c[2] = center_of(a.z, b.z);
            pr = pred(p, c);
        }
        const uint32_t m = __ballot_sync(kFull, pr);
        const uint32_t vm = __ballot_sync(kFull, valid);
        if (valid) {
            const uint32_t dst = pr ? s + lt_run + __popc(m & below)
                                    : s + n_lt_expect + gt_run + __popc(vm & ~m & below);
            if (dst < s + n) S.idx[ib ^ 1u][dst] = static_cast<uint16_t>(r);
            grow_keys12(k, pr, c);
            if (clt) *bad |= !box_contains2(clt, cgt, pr, c[0], c[1], c[2]);
        }
        lt_run += __popc(m);
        gt_run += __popc(vm & ~m);
    }
    __syncwarp();
    return lt_run;
}

__device__ __forceinline__ void warp_reduce_keys12(uint32_t* k) {
#pragma unroll
    for (int q = 0; q < 12; ++q)
        k[q] = ((q % 6) < 3) ? __reduce_min_sync(kFull, k[q]) : __reduce_max_sync(kFull, k[q]);
}

// The learned form at one binned node of the medium phase (warp-uniform):
//  * with LN.samples: write a training sample (node features, the exact
//    full-sweep optimum's axis and 1/16 position bucket, whether it beats the
//    plain split, n, both costs, the node's start);
//  * with LN.w: run the network, score 16 thresholds inside each of its two
//    best (axis, bucket) proposals exactly (one per lane), and replace the
//    plain split when the best of them costs strictly less.
#ifndef MGBVH_LEARNED_NODE_INLINE
#define MGBVH_LEARNED_NODE_INLINE 0  // 1: inline the learned form's node code into the subtree CTA (tuning knob)
#endif
#if MGBVH_LEARNED_NODE_INLINE
#define MGBVH_LEARNED_NODE_ATTR __forceinline__
#else
#define MGBVH_LEARNED_NODE_ATTR __noinline__
#endif
template <class MS>
__device__ MGBVH_LEARNED_NODE_ATTR void learned_node(const MS& S, const Learn& LN, const Params& P,
                                          const MNode& nd, uint32_t ib, uint32_t base, uint32_t s,
                                          uint32_t n, uint32_t depth, uint32_t tbase,
                                          const uint32_t* cnt, const float* ext,
                                          uint32_t plain_ck, uint32_t lane, Cand& win,
                                          uint32_t& axis, uint32_t& n_lt, bool& use_thr,
                                          uint32_t* wb) {
    float f[24];
    node_features(nd.b, nd.cb, n, depth, cnt, f);
    const float sa_p = surface_area6(nd.b);
    auto fetch = [&](uint32_t j, float* lo, float* hi) {
        const uint32_t r = S.idx[ib][s + j];
        const float4 a = S.rlo[r], b = S.rhi[r];
        lo[0] = a.x;
        lo[1] = a.y;
        lo[2] = a.z;
        hi[0] = b.x;
        hi[1] = b.y;
        hi[2] = b.z;
    };
    if (LN.samples) {
        // full sweep: every centroid a threshold on every axis; first minimum
        // of (cost, axis, threshold value)
        uint32_t bk = kNoKey, ba = 3, bt = kNoKey;
        float bthr = 0.0f;
        for (uint32_t a = 0; a < 3; ++a) {
            for (uint32_t k0 = 0; k0 < n; k0 += 32) {
                const uint32_t k = k0 + lane;
                float thr = 0.0f;
                if (k < n) {
                    float lo[3], hi[3];
                    fetch(k, lo, hi);
                    thr = center_of(lo[a], hi[a]);
                }
                Cand c;
                score_threshold(fetch, n, a, thr, k < n, sa_p, P, c, 0);
                const uint32_t ck = static_cast<uint32_t>(c.key >> 32);
                const uint32_t tk = fkey(thr);
                if (c.key != ~0ull && (ck < bk || (ck == bk && (a < ba || (a == ba && tk < bt))))) {
                    bk = ck;
                    ba = a;
                    bt = tk;
                    bthr = thr;
                }
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const uint32_t ok = __shfl_xor_sync(kFull, bk, off);
            const uint32_t oa = __shfl_xor_sync(kFull, ba, off);
            const uint32_t ot = __shfl_xor_sync(kFull, bt, off);
            const float oth = __shfl_xor_sync(kFull, bthr, off);
            if (ok < bk || (ok == bk && (oa < ba || (oa == ba && ot < bt)))) {
                bk = ok;
                ba = oa;
                bt = ot;
                bthr = oth;
            }
        }
        if (lane == 0)
            write_sample(LN, f, bk, ba, bthr, ba < 3 ? sel3(nd.cb, ba) : 0.0f, ba < 3 ? sel3(ext, ba) : 0.0f,
                         plain_ck, n, base + s - tbase);
    }
    if (LN.w && n >= LN.min_n) {
        int top0 = 0, top1 = 0;
        float refine = 0.0f;
        mgbvh_mlp::warp_forward_t(f, LN.w, lane, top0, top1, refine);
        if (!LN.gate || refine > LN.gate_thr) {
            // Interval bins (the warp's bin area is free once the binned
            // candidates are in registers): every object goes to the interval
            // of its centroid among each proposal's 16 thresholds; lane
            // p * 16 + k then scores threshold k of proposal p with lt =
            // intervals 0..k and gt = k + 1..16, the same object sets as
            // testing centroid < threshold object by object.
            uint32_t pa[2], pb[2];
            float pc[2], pe[2];
            bool act[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const uint32_t prop = (uint32_t)(q ? top1 : top0);
                pa[q] = min(prop >> 4, 2u);
                pb[q] = prop & 15u;
                pc[q] = nd.cb[pa[q]];
                pe[q] = ext[pa[q]];
                act[q] = pe[q] > 0.0f;
            }
            for (uint32_t i = lane; i < kRBinWords; i += 32) {
                const uint32_t f7 = i % 7u;
                wb[i] = f7 == 0 ? 0u : (f7 <= 3 ? kKeyPosInf : kKeyNegInf);
            }
            __syncwarp();
            // lane q * 16 + k holds threshold k of proposal q; the searches read it by shuffle
            const float lthr = proposal_threshold((lane >> 4) ? pc[1] : pc[0], (lane >> 4) ? pe[1] : pe[0],
                                                  (lane >> 4) ? pb[1] : pb[0], lane & 15u);
            for (uint32_t j0 = 0; j0 < n; j0 += 32) {  // warp-uniform trip count
                const uint32_t j = j0 + lane;
                const bool valid = j < n;
                float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
                if (valid) fetch(j, lo, hi);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (!act[q]) continue;  // warp-uniform
                    const float c = center_of(lo[pa[q]], hi[pa[q]]);
                    uint32_t a = 0, b = 16;  // interval = number of thresholds thr with !(c < thr)
#pragma unroll
                    for (int it = 0; it < 5; ++it) {
                        const uint32_t mid = min((a + b) >> 1, 15u);
                        const float tm = __shfl_sync(kFull, lthr, q * 16 + mid);
                        if (a < b) {
                            if (!(c < tm))
                                a = mid + 1;
                            else
                                b = mid;
                        }
                    }
                    if (!valid) continue;
                    uint32_t* w = wb + (q * 17 + a) * 7;
                    atomicAdd(w, 1u);
                    atomicMin(w + 1, fkey(lo[0]));
                    atomicMin(w + 2, fkey(lo[1]));
                    atomicMin(w + 3, fkey(lo[2]));
                    atomicMax(w + 4, fkey(hi[0]));
                    atomicMax(w + 5, fkey(hi[1]));
                    atomicMax(w + 6, fkey(hi[2]));
                }
            }
            __syncwarp();
            const uint32_t q = lane >> 4, k = lane & 15u;
            const uint32_t qa = q ? pa[1] : pa[0];
            const float thr = proposal_threshold(q ? pc[1] : pc[0], q ? pe[1] : pe[0], q ? pb[1] : pb[0], k);
            const uint32_t* rb = wb + q * 17u * 7u;
            Cand c;
            box_empty(c.lt);
            box_empty(c.gt);
            uint32_t nl = 0, ng = 0;
            for (uint32_t j = 0; j < 17; ++j) {
                const uint32_t* bj = rb + j * 7;
                const uint32_t cj = bj[0];
                if (cj == 0) continue;
                if (j <= k) {
                    nl += cj;
                    box_grow(c.lt, funkey(bj[1]), funkey(bj[2]), funkey(bj[3]), funkey(bj[4]),
                             funkey(bj[5]), funkey(bj[6]));
                } else {
                    ng += cj;
                    box_grow(c.gt, funkey(bj[1]), funkey(bj[2]), funkey(bj[3]), funkey(bj[4]),
                             funkey(bj[5]), funkey(bj[6]));
                }
            }
            __syncwarp();  // the interval bins are read before the warp's next use of its bin area
            c.key = ~0ull;
            c.n_lt = nl;
            c.thr = thr;
            if ((q ? act[1] : act[0]) && nl >= P.min_leaf && ng >= P.min_leaf)
                c.key = cand_key(split_cost(surface_area6(c.lt), surface_area6(c.gt), sa_p, nl, ng), qa,
                                 lane);
            const uint64_t wk2 = warp_min_key(c.key);
            const uint32_t wlo = static_cast<uint32_t>(wk2);
            if (wlo != kNoKey && static_cast<uint32_t>(wk2 >> 32) < plain_ck) {
                shfl_cand(c, wlo & 0xFFu);
                win = c;
                axis = (wlo >> 8) & 3u;
                n_lt = c.n_lt;
                use_thr = true;
            }
        }
    }
}

// The builder's transposed copy of the network parameters (layout in
// mgbvh_mlp.cuh); padding outputs are zero.
__global__ void transpose_weights_kernel(const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mgbvh_mlp::kTParams) return;
    const int src = mgbvh_mlp::transposed_source(i);
    t[i] = src >= 0 ? w[src] : __float2bfloat16_rn(0.0f);
}

// One CTA builds the subtree of one medium node (33..1024 objects).
// kQueue (the persistent batched build): records are read through L2 only,
// and each subtree of <= 32 objects is built at once by the warp that split
// it off, from shared memory, instead of going to the small list.
template <bool kLearn, class MS, bool kQueue = false, bool kSmallLevels = true>
__device__ __forceinline__ void medium_task(MS& S, const Task t, Rec* rec0, Rec* rec1,
                                            Task* small, uint32_t cap_small, const Params& P,
                                            const Out& O, const Learn& LN) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    Rec* src = (t.buf ? rec1 : rec0) + t.start;
    const uint32_t base = t.start;
    uint32_t k[12];
    init_key12(k);
    if (threadIdx.x < 12) S.rootk[threadIdx.x] = ((threadIdx.x % 6) < 3) ? kKeyPosInf : kKeyNegInf;
    if (threadIdx.x < 2) S.list_n[threadIdx.x] = 0;
    if constexpr (kQueue) {
        if (threadIdx.x == 0) S.sref_n = 0;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < t.len; i += blockDim.x) {
        const Rec r = load_rec<kQueue>(src + i);
        S.rlo[i] = r.lo;
        S.rhi[i] = r.hi;
        S.idx[0][i] = static_cast<uint16_t>(i);
        accum_keys(k, r.lo.x, r.lo.y, r.lo.z, r.hi.x, r.hi.y, r.hi.z);
    }
    // root centroid bounds (keys 6..11)
#pragma unroll
    for (int q = 6; q < 12; ++q) {
        const bool is_min = q < 9;
        const uint32_t v = is_min ? __reduce_min_sync(kFull, k[q]) : __reduce_max_sync(kFull, k[q]);
        if (lane == 0) {
            if (is_min)
                atomicMin(&S.rootk[q], v);
            else
                atomicMax(&S.rootk[q], v);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        MNode& r = S.list[0][0];
        for (int a = 0; a < 3; ++a) {
            r.b[a] = t.lo[a];
            r.b[3 + a] = t.hi[a];
            r.cb[a] = funkey(S.rootk[6 + a]);
            r.cb[3 + a] = funkey(S.rootk[9 + a]);
        }
        r.s = 0;
        r.n = t.len;
        r.slot = t.slot;
        r.pair = t.pair;
        S.list_x[0][0].depth = t.depth;
        S.list_x[0][0].ib = 0;
        S.list_n[0] = 1;
    }
    uint32_t cur = 0;
    uint32_t hmax = 0;
    bool any_split = false;
    uint32_t n_median = 0;
    for (;;) {
        __syncthreads();
        const uint32_t ncur = S.list_n[cur];
        if (ncur == 0) break;
        if (threadIdx.x == 0) S.list_n[cur ^ 1u] = 0;
        __syncthreads();
        for (uint32_t li = warp; li < ncur; li += kMediumWarps) {
            const MNode nd = S.list[cur][li];
            const MNodeExtra nx = S.list_x[cur][li];
            const uint32_t s = nd.s, n = nd.n, depth = nx.depth, ib = nx.ib;
            bool leaf = depth == P.max_depth || (n <= P.max_leaf && n < 2u * P.min_leaf);
            Cand win;
            uint32_t axis = 0, sbin = 0, n_lt = 0;
            bool median = false;
            bool use_thr = false;  // the learned form replaced the binned split
            const uint32_t B = P.bins ? P.bins : 32u;
            float ext[3];
            bool axis_ok[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                ext[a] = __fsub_rn(nd.cb[3 + a], nd.cb[a]);
                axis_ok[a] = !(ext[a] == 0.0f);
            }
            if (!leaf) {
                uint32_t* wb = S.bins[warp];
                init_task_bins(wb, lane, 32);
                __syncwarp();
                for (uint32_t p = s + lane; p < s + n; p += 32) {
                    const uint32_t r = S.idx[ib][p];
                    const float4 lo = S.rlo[r], hi = S.rhi[r];
                    const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        if (!axis_ok[a]) continue;
                        const uint32_t b = bin_of(center_of(l[a], h[a]), nd.cb[a], ext[a], B);
                        uint32_t* bw = wb + (a * 32 + b) * 7;
                        atomicAdd(bw, 1u);
                        atomicMin(bw + 1, fkey(l[0]));
                        atomicMin(bw + 2, fkey(l[1]));
                        atomicMin(bw + 3, fkey(l[2]));
                        atomicMax(bw + 4, fkey(h[0]));
                        atomicMax(bw + 5, fkey(h[1]));
                        atomicMax(bw + 6, fkey(h[2]));
                    }
                }
                __syncwarp();
                uint32_t cnt[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) cnt[a] = wb[(a * 32 + lane) * 7];
                // each axis's bin read from the warp's bins as the sweep
                // reaches it (fewer live registers)
                Cand best;
                binned_candidates_f(
                    [&](uint32_t a, uint32_t& ca, float* ba) {
                        const uint32_t* bw = wb + (a * 32 + lane) * 7;
                        ca = bw[0];
#pragma unroll
                        for (int i = 0; i < 6; ++i) ba[i] = funkey(bw[1 + i]);
                    },
                    axis_ok, B, n, surface_area6(nd.b), P, lane, best);
                const uint64_t wk = warp_min_key(best.key);
                const uint32_t wlo = static_cast<uint32_t>(wk);
                if (wlo == kNoKey) {
                    if (n > P.max_leaf)
                        median = true;
                    else
                        leaf = true;
                } else {
                    axis = (wlo >> 8) & 3u;
                    sbin = wlo & 0xFFu;
                    win = best;
                    shfl_cand(win, sbin);
                    const float cost = funkey(static_cast<uint32_t>(wk >> 32));
                    if (n <= P.max_leaf && cost >= leaf_cost(n)) leaf = true;
                    n_lt = win.n_lt;
                    if constexpr (kLearn) {
                        if (!leaf && (LN.w || LN.samples) && B == 32u)
                            learned_node(S, LN, P, nd, ib, base, s, n, depth, t.tbase, cnt, ext,
                                         static_cast<uint32_t>(wk >> 32), lane, win, axis, n_lt,
                                         use_thr, S.bins[warp]);
                        if (use_thr && lane == 0) atomicAdd(&O.ctr->learned, 1u);
                    }
                }
            }
            if (leaf) {
                medium_leaf(S, ib, base, s, n, nd.slot, depth, nd.b, t.nbase, t.tbase, P, O, lane);
                continue;
            }
            uint32_t ck[12];
            init_key12(ck);
            uint32_t ob = ib ^ 1u;
            // containment of centroids in child bounds (bvh/src/lib.rs:637-646),
            // checked on the pass that places each object
            bool bad = false;
            if (!median) {
                const float cmin = sel3(nd.cb, axis), ex = sel3(ext, axis), thr = win.thr;
                const bool by_thr = use_thr;
                const uint32_t got = medium_partition(
                    S, ib, s, n, n_lt, lane,
                    [&](uint32_t, const float* c) {
                        const float ca = sel3(c, axis);
                        return by_thr ? ca < thr : bin_of(ca, cmin, ex, B) < sbin;
                    },
                    ck, win.lt, win.gt, &bad);
                if (got != n_lt && lane == 0) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteCount);
            } else {
                // median_split on axes 0, 1, 2 over the same list (bvh/src/lib.rs:444-491,
                // 528-530): stable selection of the n/2 smallest centroid keys.
                const uint32_t m = n / 2u;
                uint32_t cb = ib;
                uint32_t best_ck = 0;
                for (uint32_t a = 0; a < 3; ++a) {
                    uint32_t dummy[12];
                    init_key12(dummy);
                    medium_partition(
                        S, cb, s, n, m, lane,
                        [&](uint32_t p, const float* c) {
                            const uint32_t key = fkey(sel3(c, a));
                            uint32_t rank = 0;
                            for (uint32_t q = s; q < s + n; ++q) {
                                const uint32_t r = S.idx[cb][q];
                                const uint32_t kq = fkey(center_of(
                                    a == 0 ? S.rlo[r].x : (a == 1 ? S.rlo[r].y : S.rlo[r].z),
                                    a == 0 ? S.rhi[r].x : (a == 1 ? S.rhi[r].y : S.rhi[r].z)));
                                rank += (kq < key || (kq == key && q < p)) ? 1u : 0u;
                            }
                            return rank < m;
                        },
                        dummy);
                    cb ^= 1u;
                    float blt[6], bgt[6];
                    box_empty(blt);
                    box_empty(bgt);
                    for (uint32_t p = s + lane; p < s + n; p += 32) {
                        const uint32_t r = S.idx[cb][p];
                        const float4 lo = S.rlo[r], hi = S.rhi[r];
                        box_grow2(blt, bgt, p < s + m, lo.x, lo.y, lo.z, hi.x, hi.y, hi.z);
                    }
                    for (int i = 0; i < 3; ++i) {
                        blt[i] = funkey(__reduce_min_sync(kFull, fkey(blt[i])));
                        bgt[i] = funkey(__reduce_min_sync(kFull, fkey(bgt[i])));
                        blt[3 + i] = funkey(__reduce_max_sync(kFull, fkey(blt[3 + i])));
                        bgt[3 + i] = funkey(__reduce_max_sync(kFull, fkey(bgt[3 + i])));
                    }
                    const float cost = split_cost(surface_area6(blt), surface_area6(bgt),
                                                  surface_area6(nd.b), m, n - m);
                    const uint32_t key = fkey(cost);
                    if (a == 0 || key < best_ck) {
                        best_ck = key;
                        for (int i = 0; i < 6; ++i) {
                            win.lt[i] = blt[i];
                            win.gt[i] = bgt[i];
                        }
                    }
                }
                ob = cb;
                n_lt = m;
                n_median++;
                for (uint32_t p = s + lane; p < s + n; p += 32) {
                    const uint32_t r = S.idx[ob][p];
                    const float4 lo = S.rlo[r], hi = S.rhi[r];
                    const float c[3] = {center_of(lo.x, hi.x), center_of(lo.y, hi.y), center_of(lo.z, hi.z)};
                    grow_keys12(ck, p < s + m, c);
                    bad |= !box_contains2(win.lt, win.gt, p < s + m, c[0], c[1], c[2]);
                }
            }
            if (__any_sync(kFull, bad) && lane == 0) set_error(O.ctr, MGBVH_ERR_ASSERT, kSiteContain);
            warp_reduce_keys12(ck);
            warp_store_node(O, t.nbase + nd.slot, nd.b, base + s - t.tbase, n, nd.pair, lane);
            any_split = true;
            hmax = max(hmax, depth);
            const uint32_t n_gt = n - n_lt;
#pragma unroll  // constant c: the child's box and keys stay in registers
            for (int c = 0; c < 2; ++c) {
                const uint32_t len = c == 0 ? n_gt : n_lt;
                const uint32_t cs = c == 0 ? s + n_lt : s;
                const uint32_t slot = c == 0 ? nd.pair : nd.pair + 1u;
                const uint32_t pair = c == 0 ? nd.pair + 2u : nd.pair + 2u * n_gt;
                const uint32_t cdepth = depth + 1u;
                const float* cbx = c == 0 ? win.gt : win.lt;
                const uint32_t* cck = c == 0 ? ck + 6 : ck;
                const bool cleaf =
                    len <= 1u || cdepth == P.max_depth || (len <= P.max_leaf && len < 2u * P.min_leaf);
                if (cleaf) {
                    medium_leaf(S, ob, base, cs, len, slot, cdepth, cbx, t.nbase, t.tbase, P, O, lane);
                } else if (len > kSmallMax) {
                    uint32_t li2 = 0;
                    if (lane == 0) li2 = atomicAdd(&S.list_n[cur ^ 1u], 1u);
                    li2 = __shfl_sync(kFull, li2, 0);
                    if (lane == 0) {
                        MNode& q = S.list[cur ^ 1u][li2];
                        for (int i = 0; i < 6; ++i) {
                            q.b[i] = cbx[i];
                            q.cb[i] = funkey(cck[i]);
                        }
                        q.s = cs;
                        q.n = len;
                        q.slot = slot;
                        q.pair = pair;
                        S.list_x[cur ^ 1u][li2].depth = cdepth;
                        S.list_x[cur ^ 1u][li2].ib = ob;
                    }
                } else {
                    if constexpr (kQueue) {
                        // the persistent build: listed, and built from shared memory
                        // once the CTA's own nodes are done
                        uint32_t ri = 0;
                        if (lane == 0) ri = atomicAdd(&S.sref_n, 1u);
                        ri = __shfl_sync(kFull, ri, 0);
                        if (lane == 0) {
                            SmallRef& q = S.sref[ri];
                            for (int i = 0; i < 6; ++i) q.b[i] = cbx[i];
                            q.slot = slot;
                            q.pair = pair;
                            q.depth = cdepth;
                            q.cs = static_cast<uint16_t>(cs);
                            q.len = static_cast<uint8_t>(len);
                            q.ob = static_cast<uint8_t>(ob);
                        }
                        continue;
                    }
                    // subtree of <= 32 objects: write its records back to this task's
                    // range of the record buffer and queue it for small_kernel
                    if (lane < len) {
                        const uint32_t r = S.idx[ob][cs + lane];
                        Rec rr;
                        rr.lo = S.rlo[r];
                        rr.hi = S.rhi[r];
                        src[cs + lane] = rr;
                    }
                    uint32_t si = 0;
                    if (lane == 0) si = atomicAdd(&O.ctr->n_small, 1u);
                    si = __shfl_sync(kFull, si, 0);
                    if (si >= cap_small) {
                        if (lane == 0) set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
                    } else if (lane == 0) {
                        Task st;
                        for (int a = 0; a < 3; ++a) {
                            st.lo[a] = cbx[a];
                            st.hi[a] = cbx[3 + a];
                        }
                        st.start = base + cs;
                        st.len = len;
                        st.slot = slot;
                        st.pair = pair;
                        st.depth = cdepth;
                        st.buf = t.buf;
                        st.tile0 = st.ntiles = 0;
                        st.nbase = t.nbase;
                        st.tbase = t.tbase;
                        small[si] = st;
                    }
                }
            }
        }
        cur ^= 1u;
    }
    if (lane == 0) {
        if (any_split) atomicMax(&O.ctr->height, hmax);
        if (n_median) atomicAdd(&O.ctr->median_splits, n_median);
    }
    if constexpr (kQueue) {
        // the subtrees of <= 32 objects, one warp each (the loop above ends
        // after a barrier, so the list is complete)
        const uint32_t ns = S.sref_n;
        for (uint32_t i = warp; i < ns; i += kMediumWarps) {
            const SmallRef q = S.sref[i];
            float slo[3] = {0.f, 0.f, 0.f}, shi[3] = {0.f, 0.f, 0.f};
            uint32_t sid = 0;
            if (lane < q.len) {
                const uint32_t r = S.idx[q.ob][q.cs + lane];
                const float4 a = S.rlo[r], b = S.rhi[r];
                slo[0] = a.x;
                slo[1] = a.y;
                slo[2] = a.z;
                sid = __float_as_uint(a.w);
                shi[0] = b.x;
                shi[1] = b.y;
                shi[2] = b.z;
            }
            if constexpr (kSmallLevels)
                warp_build_subtree_levels(slo, shi, sid, q.len, base + q.cs, q.slot, q.pair, q.depth, t.nbase,
                                          t.tbase, q.b, P, O, S.xchg[warp]);
            else
                warp_build_subtree(slo, shi, sid, q.len, base + q.cs, q.slot, q.pair, q.depth, t.nbase, t.tbase, q.b,
                                   P, O, S.xchg[warp]);
        }
    }
}

// kLearn: with the learned form's hook (network proposals, training samples);
// plain builds run the instantiation without it.
#ifndef MGBVH_MEDIUM_LEARN_CTAS
#define MGBVH_MEDIUM_LEARN_CTAS 4  // learned-form subtree CTAs per SM the register budget must allow (tuning knob)
#endif

#ifndef MGBVH_SMALL_TAKE
#define MGBVH_SMALL_TAKE 1  // 1: small-subtree warps take tasks from a counter (0: grid-stride order)
#endif
#ifndef MGBVH_MEDIUM_TAKE
#define MGBVH_MEDIUM_TAKE 1  // 1: subtree CTAs take tasks from a counter (0: grid-stride order)
#endif

// The subtree CTA's dynamic shared memory.
template <bool kLearn, uint32_t kCap>
constexpr size_t medium_smem_bytes() {
    return sizeof(MediumSmemT<kCap>);
}

template <bool kLearn, uint32_t kCap>
__global__ void __launch_bounds__(kMediumThreads, kLearn ? MGBVH_MEDIUM_LEARN_CTAS : MGBVH_MEDIUM_SMALL_CTAS)
    medium_kernel(const Task* __restrict__ tasks,
                                                                Rec* rec0, Rec* rec1, Task* small,
                                                                uint32_t cap_small, Params P, Out O,
                                                                Learn LN, const uint32_t* range) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MediumSmemT<kCap>& S = *reinterpret_cast<MediumSmemT<kCap>*>(smem_raw);
    // range (nullable): tasks [range[0], range[1]) instead of all of them
    // (range is ctr->mrange + c for slot chunk c). CTAs take the tasks in
    // turn from a counter (subtree sizes vary, so a fixed assignment leaves
    // a tail): medium_take, or mtake[c] for a chunk.
    const uint32_t t0 = range ? range[0] : 0u;
    const uint32_t n_tasks = range ? range[1] : *reinterpret_cast<volatile uint32_t*>(&O.ctr->n_medium);
    if (MGBVH_MEDIUM_TAKE) {
        __shared__ uint32_t s_ti;
        uint32_t* take = range ? O.ctr->mtake + (range - O.ctr->mrange) : &O.ctr->medium_take;
        for (;;) {
            __syncthreads();  // the previous task's readers of s_ti and of S are done
            if (threadIdx.x == 0) s_ti = t0 + atomicAdd(take, 1u);
            __syncthreads();
            const uint32_t ti = s_ti;
            if (ti >= n_tasks) break;
            medium_task<kLearn>(S, tasks[ti], rec0, rec1, small, cap_small, P, O, LN);
        }
    } else {
        for (uint32_t ti = t0 + blockIdx.x; ti < n_tasks; ti += gridDim.x) {
            __syncthreads();
            medium_task<kLearn>(S, tasks[ti], rec0, rec1, small, cap_small, P, O, LN);
        }
    }
}

// ---------------------------------------------------------------- streamed output

// The slot chunk of a subtree: the chunk of its children pair.
__device__ __forceinline__ uint32_t task_chunk(const Task& t, uint32_t slots) {
    return stream_chunk(t.nbase + t.pair, slots);
}

// A subtree's root node as its builder writes it when the root splits (one
// object per leaf: every queued subtree splits at its root).
__device__ __forceinline__ void write_task_root(const Out& O, const Task& t) {
    const float b[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
    lane_store_node(O, t.nbase + t.slot, b, t.start - t.tbase, t.len, t.pair);
}

// Subtree CTA tasks: counts per slot chunk and writes each root node, so
// that a chunk's launch writes only slots from its subtrees' children pairs
// on.
__global__ void __launch_bounds__(256) medium_count_kernel(const Task* __restrict__ tasks, Out O,
                                                           uint32_t slots) {
    pdl_enter();
    const uint32_t n = O.ctr->n_medium;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Task t = tasks[i];
        atomicAdd(&O.ctr->mbk[task_chunk(t, slots)], 1u);
        write_task_root(O, t);
    }
}

// Sorts the subtree CTA tasks by slot chunk into `out`; chunk c's tasks land
// in [mrange[c], mrange[c + 1]). Order within a chunk is free: every subtree
// writes its own slots.
__global__ void __launch_bounds__(256) medium_sort_kernel(const Task* __restrict__ in, Task* __restrict__ out,
                                                          Counters* __restrict__ ctr, uint32_t slots) {
    pdl_enter();
    uint32_t off[kStreamChunks + 1];
    off[0] = 0;
#pragma unroll
    for (uint32_t c = 0; c < kStreamChunks; ++c) off[c + 1] = off[c] + ctr->mbk[c];
    const uint32_t n = ctr->n_medium;
    if (blockIdx.x == 0 && threadIdx.x <= kStreamChunks) {
#pragma unroll
        for (uint32_t c = 0; c <= kStreamChunks; ++c)
            if (threadIdx.x == c) ctr->mrange[c] = min(off[c], n);
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Task t = in[i];
        const uint32_t c = task_chunk(t, slots);
        uint32_t base = 0;
#pragma unroll
        for (uint32_t q = 0; q < kStreamChunks; ++q)
            if (q == c) base = off[q];
        const uint32_t pos = base + atomicAdd(&ctr->mbcur[c], 1u);
        if (pos < n)
            out[pos] = t;
        else
            set_error(ctr, MGBVH_ERR_ASSERT, kSiteCount);  // counts agree by construction
    }
}

// Appends the subtrees of <= 32 objects of slot chunk c (all queued once
// chunk c's subtree CTAs ran) to `out`, and writes the root node of every
// subtree whose root slot lies in chunk c (all queued by then too: a root
// slot lies in the block of the subtree CTA or level pass that queued it).
// A root can lie in an earlier chunk than its children pair, so roots are
// written by the chunk that holds them, before that chunk is copied. The
// CTA that finishes last records the end of the chunk's range, srange[c + 1]
// (srange[c] is the previous chunk's end).
__global__ void __launch_bounds__(256) small_select_kernel(const Task* __restrict__ in, Task* __restrict__ out,
                                                           uint32_t cap, Out O, uint32_t c, uint32_t slots) {
    pdl_enter();
    __shared__ uint32_t last;
    Counters* ctr = O.ctr;
    const uint32_t n = ctr->n_small;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Task t = in[i];
        if (stream_chunk(t.nbase + t.slot, slots) == c) write_task_root(O, t);
        if (task_chunk(t, slots) != c) continue;
        const uint32_t pos = atomicAdd(&ctr->s2n, 1u);
        if (pos < cap)
            out[pos] = t;
        else
            set_error(ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&ctr->sdone[c], 1u) == gridDim.x - 1u ? 1u : 0u;
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        ctr->srange[c + 1] = min(*reinterpret_cast<volatile uint32_t*>(&ctr->s2n), cap);
    }
}

// ---------------------------------------------------------------- small

// One warp per subtree of <= 32 objects. kLevels: the level-synchronous
// builder (every node adaptive with one threshold per object); otherwise the
// depth-first builder that also covers binned nodes and fixed step counts.
// kMinBlocks: CTAs of 256 threads per SM the register budget allows (the
// context's small-subtree occupancy): 3 (80 registers, 24 warps per SM) or 2
// (126 registers, 16 warps). The kernel is issue-bound on fixed-latency
// dependencies; on the noisy icosphere the extra warps hide more of them than
// the spills of the tighter budget add (warp-subtree phase 0.568 -> 0.543 ms;
// 4 CTAs at 64 registers: 0.594 ms), while the batched scene builds 3% faster
// at 16 warps. The autotuner picks it per workload.
template <bool kLevels, int kMinBlocks>
// range (nullable): build tasks [range[0], range[1]) instead of all of them.
__global__ void __launch_bounds__(256, kMinBlocks) small_kernel(const Task* __restrict__ tasks,
                                                   const Rec* __restrict__ rec0,
                                                   const Rec* __restrict__ rec1, Params P, Out O,
                                                   const uint32_t* range) {
    pdl_enter();
    __shared__ XRec xchg[8][32];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t w0 = range ? range[0] : 0u;
    const uint32_t n_tasks = range ? range[1] : *reinterpret_cast<volatile uint32_t*>(&O.ctr->n_small);
    const uint32_t wpb = blockDim.x >> 5;  // warps per CTA (64..256 threads)
    // warps take tasks in turn from a counter (subtree sizes vary, so a
    // fixed assignment leaves a tail): small_take, or stake[c] for slot
    // chunk c (range is ctr->srange + c)
    uint32_t* take = range ? O.ctr->stake + (range - O.ctr->srange) : &O.ctr->small_take;
    uint32_t w = w0 + blockIdx.x * wpb + wib;
    for (;; w += gridDim.x * wpb) {
        if (MGBVH_SMALL_TAKE) {
            uint32_t tw = 0;
            if (lane == 0) tw = w0 + atomicAdd(take, 1u);
            w = __shfl_sync(kFull, tw, 0);
        }
        if (w >= n_tasks) break;
        const Task t = tasks[w];
        const Rec* src = (t.buf ? rec1 : rec0) + t.start;
        float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
        uint32_t id = 0;
        if (lane < t.len) {
            const Rec r = src[lane];
            lo[0] = r.lo.x;
            lo[1] = r.lo.y;
            lo[2] = r.lo.z;
            id = __float_as_uint(r.lo.w);
            hi[0] = r.hi.x;
            hi[1] = r.hi.y;
            hi[2] = r.hi.z;
        }
        const float b[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
        if constexpr (kLevels)
            warp_build_subtree_levels(lo, hi, id, t.len, t.start, t.slot, t.pair, t.depth, t.nbase,
                                      t.tbase, b, P, O, xchg[wib]);
        else
            warp_build_subtree(lo, hi, id, t.len, t.start, t.slot, t.pair, t.depth, t.nbase, t.tbase,
                               b, P, O, xchg[wib]);
    }
}

// ---------------------------------------------------------------- persistent batched build
//
// A batch of meshes (every BLAS and the TLAS) built by one persistent launch
// that takes node tasks from a device-side queue, in place of the level
// passes and the subtree launches. One CTA of kMediumThreads threads per
// resident slot loops: take a task, build it, push its children.
//   above medium_max   the CTA bins the node (3 x 32 bins in shared memory),
//                      warp 0 picks the split, the CTA partitions the records
//                      stably into the other buffer and pushes the children;
//   33..medium_max     the CTA builds the whole subtree in shared memory
//                      (medium_task), its warps building each subtree of <= 32
//                      objects as soon as they split it off;
//   <= 32              (children of the nodes above medium_max) warp 0 builds it.
// Tickets: a CTA takes the next ticket with one atomicAdd on the head (no
// retries under contention) and waits for entry `ticket` to be marked ready,
// or for the pending count to reach 0 (every task finished: the batch is
// built, tickets past the last push are never filled, and the CTA leaves). A
// push counts its task as pending, reserves the next entry, writes it, fences
// and marks it ready; a finished task is uncounted after its children were
// pushed. Every wait is bounded by a deadline on the global timer; when one
// runs out the CTA records the time-out, raises abort and leaves, and so do
// all others at their next poll: the launch ends with MGBVH_ERR_TIMEOUT.
// Nodes that need the forced median are queued for the median passes, which
// run after the launch as in the level-pass build.

constexpr uint32_t kQueueMaxMesh = 1u << 22;  // largest mesh the persistent build takes (objects)
#ifndef MGBVH_QUEUE_MIN_BLOCKS
#define MGBVH_QUEUE_MIN_BLOCKS 3  // persistent CTAs per SM the register budget must allow (tuning knob)
#endif

struct QueueState {
    uint32_t head, tail;  // next ticket to hand out, next entry to reserve
    uint32_t pad0;
    uint32_t pending;     // tasks pushed and not yet finished
    uint32_t abort;       // an error or a time-out: every CTA leaves
    uint32_t timeouts;    // waits that ran out
    uint32_t pad[2];
};

struct QueueArgs {
    Task* q;           // queue entries
    uint32_t* qready;  // 1 once entry i is written
    uint32_t* qcb;     // centroid bound keys of entry i (6; level-pass-size nodes)
    uint32_t qcap;
    QueueState* st;
    Task* med;         // nodes waiting for the forced median (count in ctr->n_med)
    uint32_t med_cap;
    unsigned long long wait_ns;  // longest wait before a time-out
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t vload(const uint32_t* p) { return *reinterpret_cast<const volatile uint32_t*>(p); }

__device__ __forceinline__ void queue_abort(const QueueArgs& Q) { atomicExch(&Q.st->abort, 1u); }

// One thread: push a node task (cb: its centroid bound keys when it is above
// medium_max).
__device__ void queue_push_main(const QueueArgs& Q, const Task& t, const uint32_t* cb, Counters* ctr) {
    atomicAdd(&Q.st->pending, 1u);
    const uint32_t i = atomicAdd(&Q.st->tail, 1u);
    if (i >= Q.qcap) {
        set_error(ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
        queue_abort(Q);
        return;
    }
    Q.q[i] = t;
    if (cb)
        for (int k = 0; k < 6; ++k) Q.qcb[6 * i + k] = cb[k];
    __threadfence();
    atomicExch(&Q.qready[i], 1u);
}

// Thread 0: the next task (kind 1: entry idx) or none (kind 0: the batch is
// done, or aborted).
struct Popped {
    uint32_t kind, idx, count;
};

__device__ Popped queue_pop(const QueueArgs& Q) {
    Popped p{0u, 0u, 0u};
    if (vload(&Q.st->abort)) return p;
    const uint32_t h = atomicAdd(&Q.st->head, 1u);
    const unsigned long long t0 = global_ns();
    uint32_t ns = 32;
    for (;;) {
        if (h < Q.qcap && vload(Q.qready + h) != 0u) {
            __threadfence();  // the entry (and the records it names) after its mark
            p.kind = 1;
            p.idx = h;
            return p;
        }
        if (vload(&Q.st->abort)) return p;
        // nothing pending: no entry will come for this ticket
        if (vload(&Q.st->pending) == 0u) return p;
        if (global_ns() - t0 > Q.wait_ns) {
            atomicAdd(&Q.st->timeouts, 1u);
            queue_abort(Q);
            return p;
        }
        __nanosleep(ns);
        ns = min(ns * 2u, 1024u);
    }
}

struct LargeSmem {
    uint32_t bins[kBinWords];
    uint32_t wlt[kMediumWarps], wn[kMediumWarps];
    uint32_t keys[12];
    uint32_t kind, axis, split_bin, n_lt;  // kind: 0 split, 1 leaf, 2 forced median
    float ltb[6], gtb[6];
    int bad;
};

// One CTA: a node above medium_max objects (records in buffer t.buf, its
// centroid bound keys cbk), as lvl_bin + lvl_eval + lvl_part do for a level.
__device__ __noinline__ void queue_large_task(const QueueArgs& Q, LargeSmem& L, const Task& t, const uint32_t* cbk, Rec* rec0,
                                 Rec* rec1, const Params& P, const Out& O) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const Rec* src = (t.buf ? rec1 : rec0) + t.start;
    Rec* dst = (t.buf ? rec0 : rec1) + t.start;
    const float nb[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
    const uint32_t n = t.len, B = P.bins ? P.bins : 32u;
    float cmn[3], ext[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        cmn[a] = funkey(__ldcg(cbk + a));
        ext[a] = __fsub_rn(funkey(__ldcg(cbk + 3 + a)), cmn[a]);
    }
    const bool leaf0 = t.depth == P.max_depth || (n <= P.max_leaf && n < 2u * P.min_leaf);
    if (!leaf0) {
        init_task_bins(L.bins, tid, blockDim.x);
        __syncthreads();
        for (uint32_t i = tid; i < n; i += blockDim.x) {
            const Rec r = ldcg_rec(src + i);
            const float l[3] = {r.lo.x, r.lo.y, r.lo.z}, h[3] = {r.hi.x, r.hi.y, r.hi.z};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (ext[a] == 0.0f) continue;  // block-uniform
                uint32_t* w = L.bins + (a * 32 + bin_of(center_of(l[a], h[a]), cmn[a], ext[a], B)) * 7;
                atomicAdd(w, 1u);
                atomicMin(w + 1, fkey(l[0]));
                atomicMin(w + 2, fkey(l[1]));
                atomicMin(w + 3, fkey(l[2]));
                atomicMax(w + 4, fkey(h[0]));
                atomicMax(w + 5, fkey(h[1]));
                atomicMax(w + 6, fkey(h[2]));
            }
        }
        __syncthreads();
    }
    if (warp == 0) {
        uint32_t kind = 1;
        if (!leaf0) {
            uint32_t cnt[3];
            float box[3][6];
            bool axis_ok[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const uint32_t* bw = L.bins + (a * 32 + lane) * 7;
                cnt[a] = bw[0];
                for (int i = 0; i < 6; ++i) box[a][i] = funkey(bw[1 + i]);
                axis_ok[a] = !(ext[a] == 0.0f);
            }
            Cand best;
            binned_candidates(cnt, box, axis_ok, B, n, surface_area6(nb), P, lane, best);
            const uint64_t wk = warp_min_key(best.key);
            const uint32_t wlo = static_cast<uint32_t>(wk);
            if (wlo == kNoKey) {
                kind = n > P.max_leaf ? 2u : 1u;
            } else {
                const uint32_t sb = wlo & 0xFFu;
                Cand win = best;
                shfl_cand(win, sb);
                kind = (n <= P.max_leaf && funkey(static_cast<uint32_t>(wk >> 32)) >= leaf_cost(n)) ? 1u : 0u;
                if (lane == 0) {
                    L.axis = (wlo >> 8) & 3u;
                    L.split_bin = sb;
                    L.n_lt = win.n_lt;
                    for (int i = 0; i < 6; ++i) {
                        L.ltb[i] = win.lt[i];
                        L.gtb[i] = win.gt[i];
                    }
                }
            }
        }
        if (lane == 0) {
            L.kind = kind;
            L.bad = 0;
        }
        if (lane < 12) L.keys[lane] = ((lane % 6) < 3) ? kKeyPosInf : kKeyNegInf;
    }
    __syncthreads();
    const uint32_t kind = L.kind;
    if (kind == 2) {  // the forced median: after the launch, by the median passes
        if (tid == 0) {
            const uint32_t mi = atomicAdd(&O.ctr->n_med, 1u);
            if (mi < Q.med_cap)
                Q.med[mi] = t;
            else
                set_error(O.ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
        }
        return;
    }
    if (kind == 1) {  // a leaf of all n objects, in list order
        if (warp == 0) warp_store_node(O, t.nbase + t.slot, nb, t.start - t.tbase, n, 0u, lane);
        for (uint32_t i = tid; i < n; i += blockDim.x) O.perm[t.start + i] = __float_as_uint(__ldcg(&src[i].lo).w);
        if (tid == 0) {
            atomicAdd(&O.ctr->holes, 1u);
            if (t.depth == P.max_depth) atomicAdd(&O.ctr->depth_capped, 1u);
        }
        return;
    }
    // stable partition: chunks of 4 records per thread; warp w holds records
    // w*128 .. w*128+127 of the chunk, 32 at a time
    const uint32_t axis = L.axis, split_bin = L.split_bin, n_lt = L.n_lt;
    const float cmin = sel3(cmn, axis), ex = sel3(ext, axis);
    const uint32_t n_gt = n - n_lt;
    const uint32_t d1 = t.depth + 1u;
    const bool leaf_lt = n_lt <= 1u || d1 == P.max_depth || (n_lt <= P.max_leaf && n_lt < 2u * P.min_leaf);
    const bool leaf_gt = n_gt <= 1u || d1 == P.max_depth || (n_gt <= P.max_leaf && n_gt < 2u * P.min_leaf);
    const uint32_t below = (1u << lane) - 1u;
    float ltb[6], gtb[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        ltb[i] = L.ltb[i];
        gtb[i] = L.gtb[i];
    }
    uint32_t k[12];
    init_key12(k);
    bool bad = false;
    uint32_t run_lt = 0, run_gt = 0;
    constexpr uint32_t kPer = 4, kChunk = kMediumThreads * kPer;
    for (uint32_t base = 0; base < n; base += kChunk) {
        Rec r[kPer];
        uint32_t bal[kPer], vm[kPer];
        uint32_t lw = 0, nw = 0;
#pragma unroll
        for (uint32_t g = 0; g < kPer; ++g) {
            const uint32_t i = base + warp * (32u * kPer) + g * 32u + lane;
            bool pred = false;
            if (i < n) {
                r[g] = ldcg_rec(src + i);
                // selects, not a run-time index into r (which would put it in local memory)
                const float la = axis == 0 ? r[g].lo.x : (axis == 1 ? r[g].lo.y : r[g].lo.z);
                const float ha = axis == 0 ? r[g].hi.x : (axis == 1 ? r[g].hi.y : r[g].hi.z);
                pred = bin_of(center_of(la, ha), cmin, ex, B) < split_bin;
            }
            bal[g] = __ballot_sync(kFull, pred);
            vm[g] = __ballot_sync(kFull, i < n);
            lw += __popc(bal[g]);
            nw += __popc(vm[g]);
        }
        if (lane == 0) {
            L.wlt[warp] = lw;
            L.wn[warp] = nw;
        }
        __syncthreads();
        uint32_t lt_before = 0, gt_before = 0, lt_tot = 0, n_tot = 0;
#pragma unroll
        for (uint32_t q = 0; q < kMediumWarps; ++q) {
            const uint32_t a = L.wlt[q], b = L.wn[q];
            lt_before += q < warp ? a : 0u;
            gt_before += q < warp ? b - a : 0u;
            lt_tot += a;
            n_tot += b;
        }
        uint32_t lt_run = run_lt + lt_before, gt_run = run_gt + gt_before;
#pragma unroll
        for (uint32_t g = 0; g < kPer; ++g) {
            const bool valid = (vm[g] >> lane) & 1u;
            if (valid) {
                const bool pred = (bal[g] >> lane) & 1u;
                const uint32_t dest = pred ? lt_run + __popc(bal[g] & below)
                                           : n_lt + gt_run + __popc(vm[g] & ~bal[g] & below);
                if (dest < n) {
                    dst[dest] = r[g];
                    if (pred ? leaf_lt : leaf_gt) O.perm[t.start + dest] = __float_as_uint(r[g].lo.w);
                } else {
                    bad = true;
                }
                const float c[3] = {center_of(r[g].lo.x, r[g].hi.x), center_of(r[g].lo.y, r[g].hi.y),
                                    center_of(r[g].lo.z, r[g].hi.z)};
                bad |= !box_contains2(ltb, gtb, pred, c[0], c[1], c[2]);
                grow_keys12(k, pred, c);
            }
            lt_run += __popc(bal[g]);
            gt_run += __popc(vm[g] & ~bal[g]);
        }
        run_lt += lt_tot;
        run_gt += n_tot - lt_tot;
        __syncthreads();  // wlt/wn are rewritten by the next chunk
    }
#pragma unroll
    for (int q = 0; q < 12; ++q) {
        const bool is_min = (q % 6) < 3;
        const uint32_t v = is_min ? __reduce_min_sync(kFull, k[q]) : __reduce_max_sync(kFull, k[q]);
        if (lane == 0) {
            if (is_min)
                atomicMin(&L.keys[q], v);
            else
                atomicMax(&L.keys[q], v);
        }
    }
    if (__any_sync(kFull, bad) && lane == 0) L.bad = 1;
    __threadfence();  // the records and leaf entries before the children are pushed
    __syncthreads();
    if (warp != 0) return;
    if (run_lt != n_lt || L.bad) {
        if (lane == 0) set_error(O.ctr, MGBVH_ERR_ASSERT, run_lt != n_lt ? kSiteCount : kSiteContain);
        return;
    }
    warp_store_node(O, t.nbase + t.slot, nb, t.start - t.tbase, n, t.pair, lane);
    if (lane == 0) atomicMax(&O.ctr->height, t.depth);
#pragma unroll
    for (int c = 0; c < 2; ++c) {  // [0] gt, [1] lt, as the reference pushes them
        const uint32_t len = c == 0 ? n_gt : n_lt;
        const uint32_t start = c == 0 ? t.start + n_lt : t.start;
        const uint32_t slot = c == 0 ? t.pair : t.pair + 1u;
        float cb[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) cb[i] = c == 0 ? gtb[i] : ltb[i];
        if (c == 0 ? leaf_gt : leaf_lt) {
            warp_store_node(O, t.nbase + slot, cb, start - t.tbase, len, 0u, lane);
            if (lane == 0 && len > 1) {
                atomicAdd(&O.ctr->holes, 1u);
                if (d1 == P.max_depth) atomicAdd(&O.ctr->depth_capped, 1u);
            }
            continue;
        }
        if (lane == 0) {
            Task ct;
            for (int a = 0; a < 3; ++a) {
                ct.lo[a] = cb[a];
                ct.hi[a] = cb[3 + a];
            }
            ct.start = start;
            ct.len = len;
            ct.slot = slot;
            ct.pair = c == 0 ? t.pair + 2u : t.pair + 2u * n_gt;
            ct.depth = d1;
            ct.buf = t.buf ^ 1u;
            ct.tile0 = ct.ntiles = 0;
            ct.nbase = t.nbase;
            ct.tbase = t.tbase;
            queue_push_main(Q, ct, len > P.medium_max ? L.keys + (c == 0 ? 6 : 0) : nullptr, O.ctr);
        }
    }
}

// The persistent build's subtree CTA and warp-subtree tasks, as separate
// (not inlined) functions: each gets its own register allocation instead of
// the union of every task kind's.
template <uint32_t kCap, bool kLevels>
__device__ __noinline__ void queue_medium_task(MediumSmemQ<kCap>& S, const Task& t, Rec* rec0, Rec* rec1,
                                               const Params& P, const Out& O) {
    medium_task<false, MediumSmemQ<kCap>, true, kLevels>(S, t, rec0, rec1, nullptr, 0u, P, O,
                                                         Learn{nullptr, 0, nullptr, 0, nullptr});
}

template <bool kLevels>
__device__ __noinline__ void queue_small_task(const Task& t, const Rec* rec0, const Rec* rec1, const Params& P,
                                              const Out& O, XRec* xchg) {
    const uint32_t lane = threadIdx.x & 31u;
    const Rec* src = (t.buf ? rec1 : rec0) + t.start;
    float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
    uint32_t id = 0;
    if (lane < t.len) {
        const Rec r = ldcg_rec(src + lane);
        lo[0] = r.lo.x;
        lo[1] = r.lo.y;
        lo[2] = r.lo.z;
        id = __float_as_uint(r.lo.w);
        hi[0] = r.hi.x;
        hi[1] = r.hi.y;
        hi[2] = r.hi.z;
    }
    const float b[6] = {t.lo[0], t.lo[1], t.lo[2], t.hi[0], t.hi[1], t.hi[2]};
    if constexpr (kLevels)
        warp_build_subtree_levels(lo, hi, id, t.len, t.start, t.slot, t.pair, t.depth, t.nbase, t.tbase, b, P, O,
                                  xchg);
    else
        warp_build_subtree(lo, hi, id, t.len, t.start, t.slot, t.pair, t.depth, t.nbase, t.tbase, b, P, O, xchg);
}

template <uint32_t kCap, bool kLevels>
__global__ void __launch_bounds__(kMediumThreads, MGBVH_QUEUE_MIN_BLOCKS)
    queue_build_kernel(QueueArgs Q, Rec* rec0, Rec* rec1, Params P, Out O) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MediumSmemQ<kCap>& S = *reinterpret_cast<MediumSmemQ<kCap>*>(smem_raw);
    LargeSmem& L = *reinterpret_cast<LargeSmem*>(smem_raw);  // the same space: one task at a time
    __shared__ Popped pop;
    const uint32_t warp = threadIdx.x >> 5;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) pop = queue_pop(Q);
        __syncthreads();
        const Popped p = pop;
        if (p.kind == 0) break;
        const Task t = ldcg_task(Q.q + p.idx);
        if (t.len > P.medium_max)
            queue_large_task(Q, L, t, Q.qcb + 6 * p.idx, rec0, rec1, P, O);
        else if (t.len > kSmallMax)
            queue_medium_task<kCap, kLevels>(S, t, rec0, rec1, P, O);
        else if (warp == 0)  // a subtree of <= 32 objects split off a node above medium_max
            queue_small_task<kLevels>(t, rec0, rec1, P, O, S.xchg[0]);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) atomicSub(&Q.st->pending, 1u);
    }
}

// ---------------------------------------------------------------- compaction

__global__ void widen_used_kernel(const uint8_t* __restrict__ used, uint32_t n, uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = used[i];
}

__global__ void compact_kernel(const mgbvh_node* __restrict__ src, const uint32_t* __restrict__ lens,
                               const uint8_t* __restrict__ used, const uint32_t* __restrict__ newidx,
                               uint32_t cap, mgbvh_node* __restrict__ dst, uint32_t* dst_lens) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < cap; s += gridDim.x * blockDim.x) {
        if (!used[s]) continue;
        mgbvh_node nd = src[s];
        if (nd.child_node) nd.child_node = newidx[nd.child_node];
        const uint32_t d = newidx[s];
        dst[d] = nd;
        if (dst_lens) dst_lens[d] = lens[s];
    }
}



// ---------------------------------------------------------------- instances

// World AABB of every instance, as marigold's scene upload computes it for
// the TLAS (marigold/src/app/data/scene/model.rs:191-234): the 8 corners of
// the instance's mesh bounds, in the order (min,min,min), (min,min,max), ...,
// (max,max,max), as (x, y, z, 1) through the column-major transform; each
// component is ((c0 x + c1 y) + c2 z) + c3 * 1 with every product and sum
// rounded on its own (glam 0.30.10 Mat4 * Vec4: the column products summed
// in column order, no fused multiply-add), then the running min/max over the
// corners in that order with a tie taking the later corner (the SSE
// minps/maxps behind Vec3A::min/max). Grid-stride over instances.
__global__ void instance_aabbs_kernel(const float* __restrict__ mesh_bounds, uint32_t mesh_count,
                                      const uint32_t* __restrict__ inst_mesh,
                                      const float* __restrict__ xf, uint32_t n,
                                      float* __restrict__ out, Counters* ctr) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t m = inst_mesh[i];
        if (m >= mesh_count) {
            set_error(ctr, MGBVH_ERR_INVALID_ARG, kSiteMeshIndex);
            continue;
        }
        const float* b = mesh_bounds + 6 * (size_t)m;
        const float* t = xf + 16 * (size_t)i;
        float lo[3], hi[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            lo[r] = __int_as_float(0x7F800000);
            hi[r] = __int_as_float(0xFF800000);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float x = b[(c >> 2) & 1 ? 3 : 0], y = b[(c >> 1) & 1 ? 4 : 1], z = b[c & 1 ? 5 : 2];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const float v = __fadd_rn(
                    __fadd_rn(__fadd_rn(__fmul_rn(t[r], x), __fmul_rn(t[4 + r], y)), __fmul_rn(t[8 + r], z)),
                    __fmul_rn(t[12 + r], 1.0f));
                lo[r] = lo[r] < v ? lo[r] : v;
                hi[r] = hi[r] > v ? hi[r] : v;
            }
        }
        float* o = out + 6 * (size_t)i;
        o[0] = lo[0];
        o[1] = lo[1];
        o[2] = lo[2];
        o[3] = hi[0];
        o[4] = hi[1];
        o[5] = hi[2];
    }
}

// ---------------------------------------------------------------- batched builds
//
// Many BVHs (the BLAS of every mesh and the TLAS over instances) in one
// pipeline: the objects of all meshes are one record array, each mesh's root
// is queued like a single build's root, and every node a kernel writes goes
// to its mesh's own node range (slots offset by nbase, start indices
// relative to the mesh's first record at tbase), so each mesh's nodes, child
// links and permutation are exactly those of a build of that mesh alone.

struct DevMesh {
    const float* verts;  // NULL for an AABB list
    const uint32_t* tris;
    const float* aabbs;
    uint32_t stride_floats, nverts;
    uint32_t n, tbase, nbase;
    uint32_t has_bounds;
    float bounds[6];
    uint32_t cls, list_index, tile0, ntiles;  // root plan (0 leaf, 1 small, 2 medium, 3 large, 4 empty)
};

__device__ __forceinline__ uint32_t mesh_of(const uint32_t* __restrict__ offs, uint32_t nm, uint32_t g) {
    uint32_t lo = 0, hi = nm;  // offs[lo] <= g < offs[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (offs[mid] <= g)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Object records of every mesh (local object ids) and per-mesh root keys
// (bounds lo/hi, centroid lo/hi; 12 per mesh).
__global__ void __launch_bounds__(256) prep_batch_kernel(const DevMesh* __restrict__ meshes,
                                                         const uint32_t* __restrict__ toffs,
                                                         uint32_t nm, uint32_t total,
                                                         Rec* __restrict__ out, uint32_t* mkeys,
                                                         Counters* ctr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    // whole warps iterate together so that same-mesh warps can reduce first
    for (uint32_t g0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; g0 < total; g0 += stride) {
        const uint32_t g = g0 + lane;
        const bool valid = g < total;
        uint32_t m = valid ? mesh_of(toffs, nm, g) : 0u;
        float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
        if (valid) {
            const DevMesh& M = meshes[m];
            const uint32_t l = g - M.tbase;
            if (M.verts) {
                uint32_t t0 = M.tris[3 * (size_t)l], t1 = M.tris[3 * (size_t)l + 1],
                         t2 = M.tris[3 * (size_t)l + 2];
                if (t0 >= M.nverts || t1 >= M.nverts || t2 >= M.nverts) {
                    set_error(ctr, MGBVH_ERR_INVALID_ARG, kSiteIndex);
                    t0 = t1 = t2 = 0;
                }
                const float* p0 = M.verts + (size_t)t0 * M.stride_floats;
                const float* p1 = M.verts + (size_t)t1 * M.stride_floats;
                const float* p2 = M.verts + (size_t)t2 * M.stride_floats;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float x0 = __fadd_rn(__ldg(p0 + a), 0.0f), x1 = __fadd_rn(__ldg(p1 + a), 0.0f),
                                x2 = __fadd_rn(__ldg(p2 + a), 0.0f);
                    lo[a] = fminf(fminf(x0, x1), x2);
                    hi[a] = fmaxf(fmaxf(x0, x1), x2);
                }
            } else {
                const float* p = M.aabbs + 6 * (size_t)l;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    lo[a] = __fadd_rn(__ldg(p + a), 0.0f);
                    hi[a] = __fadd_rn(__ldg(p + 3 + a), 0.0f);
                }
            }
            Rec r;
            r.lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(l));
            r.hi = make_float4(hi[0], hi[1], hi[2], 0.0f);
            out[g] = r;
        }
        uint32_t k[12];
        init_key12(k);
        if (valid) accum_keys(k, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
        const uint32_t m0 = __shfl_sync(kFull, m, 0);
        const bool uniform = __all_sync(kFull, !valid || m == m0);
        if (uniform) {
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                const bool is_min = (q % 6) < 3;
                const uint32_t v = is_min ? __reduce_min_sync(kFull, k[q]) : __reduce_max_sync(kFull, k[q]);
                if (lane == 0) {
                    if (is_min)
                        atomicMin(&mkeys[12 * m0 + q], v);
                    else
                        atomicMax(&mkeys[12 * m0 + q], v);
                }
            }
        } else if (valid) {
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                if ((q % 6) < 3)
                    atomicMin(&mkeys[12 * m + q], k[q]);
                else
                    atomicMax(&mkeys[12 * m + q], k[q]);
            }
        }
    }
}

__global__ void init_mkeys_kernel(uint32_t* mkeys, uint32_t nm) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 12 * nm; i += gridDim.x * blockDim.x)
        mkeys[i] = ((i % 6) < 3) ? kKeyPosInf : kKeyNegInf;
}

// One warp per mesh: queue its root (or finish it when the root is a leaf).
__global__ void init_roots_kernel(const DevMesh* __restrict__ meshes, uint32_t nm,
                                  const uint32_t* __restrict__ mkeys, Task* large, uint32_t* bins,
                                  uint32_t* cbkeys, uint32_t* tile_task, uint32_t* tile_begin,
                                  Task* medium, Task* small, Out O, uint32_t max_depth) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; m < nm; m += nwarps) {
        const DevMesh& M = meshes[m];
        if (M.cls > 3) continue;  // empty mesh: nothing to build
        float b[6];
        for (int i = 0; i < 6; ++i) b[i] = M.has_bounds ? M.bounds[i] : funkey(mkeys[12 * m + i]);
        Task t;
        for (int a = 0; a < 3; ++a) {
            t.lo[a] = b[a];
            t.hi[a] = b[3 + a];
        }
        t.start = M.tbase;
        t.len = M.n;
        t.slot = 0;
        t.pair = 1;
        t.depth = 0;
        t.buf = 0;
        t.tile0 = M.tile0;
        t.ntiles = M.ntiles;
        t.nbase = M.nbase;
        t.tbase = M.tbase;
        if (M.cls == 0) {
            warp_store_node(O, M.nbase, b, 0u, M.n, 0u, lane);
            for (uint32_t i = lane; i < M.n; i += 32) O.perm[M.tbase + i] = i;
            if (lane == 0 && M.n > 1) {
                atomicAdd(&O.ctr->holes, 1u);
                if (max_depth == 0) atomicAdd(&O.ctr->depth_capped, 1u);
            }
        } else if (M.cls == 1) {
            if (lane == 0) small[M.list_index] = t;
        } else if (M.cls == 2) {
            if (lane == 0) medium[M.list_index] = t;
        } else {
            if (lane == 0) large[M.list_index] = t;
            init_task_bins(bins + (size_t)M.list_index * kBinWords, lane, 32);
            if (lane < 6) cbkeys[6 * M.list_index + lane] = mkeys[12 * m + 6 + lane];
            for (uint32_t i = lane; i < M.ntiles; i += 32) {
                tile_task[M.tile0 + i] = M.list_index;
                tile_begin[M.tile0 + i] = i * kTile;
            }
        }
    }
}

// The batch's roots into the queues: main entries (with centroid bound keys)
// and small entries, ready flags set; leaf roots finished here.
__global__ void queue_roots_kernel(const DevMesh* __restrict__ meshes, uint32_t nm, const uint32_t* __restrict__ mkeys,
                                   QueueArgs Q, Out O, uint32_t max_depth, uint32_t medium_max, uint32_t hold) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    if (blockIdx.x == 0 && threadIdx.x == 0 && hold) atomicAdd(&Q.st->pending, hold);
    for (uint32_t m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; m < nm; m += nwarps) {
        const DevMesh& M = meshes[m];
        if (M.cls > 3) continue;  // empty mesh: nothing to build
        float b[6];
        for (int i = 0; i < 6; ++i) b[i] = M.has_bounds ? M.bounds[i] : funkey(mkeys[12 * m + i]);
        if (M.cls == 0) {
            warp_store_node(O, M.nbase, b, 0u, M.n, 0u, lane);
            for (uint32_t i = lane; i < M.n; i += 32) O.perm[M.tbase + i] = i;
            if (lane == 0 && M.n > 1) {
                atomicAdd(&O.ctr->holes, 1u);
                if (max_depth == 0) atomicAdd(&O.ctr->depth_capped, 1u);
            }
            continue;
        }
        if (lane != 0) continue;
        Task t;
        for (int a = 0; a < 3; ++a) {
            t.lo[a] = b[a];
            t.hi[a] = b[3 + a];
        }
        t.start = M.tbase;
        t.len = M.n;
        t.slot = 0;
        t.pair = 1;
        t.depth = 0;
        t.buf = 0;
        t.tile0 = t.ntiles = 0;
        t.nbase = M.nbase;
        t.tbase = M.tbase;
        queue_push_main(Q, t, M.n > medium_max ? mkeys + 12 * m + 6 : nullptr, O.ctr);
    }
}

// Compaction of a batch: slot s of mesh m moves to newidx[s] and its child
// link (local) to newidx[nbase_m + child] - newidx[nbase_m].
__global__ void compact_batch_kernel(const mgbvh_node* __restrict__ src, const uint32_t* __restrict__ lens,
                                     const uint8_t* __restrict__ used, const uint32_t* __restrict__ newidx,
                                     const uint32_t* __restrict__ noffs, uint32_t nm, uint32_t slots,
                                     mgbvh_node* __restrict__ dst, uint32_t* dst_lens) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        if (!used[s]) continue;
        const uint32_t m = mesh_of(noffs, nm, s);
        const uint32_t base_new = newidx[noffs[m]];
        mgbvh_node nd = src[s];
        if (nd.child_node) nd.child_node = newidx[noffs[m] + nd.child_node] - base_new;
        const uint32_t d = newidx[s];
        dst[d] = nd;
        if (dst_lens) dst_lens[d] = lens[s];
    }
}

// ---------------------------------------------------------------- allocation-free build
//
// Scratch of mgbvh_build_aabbs_noalloc lives in this file-scope device array,
// part of the library image: every device that loads the library holds it
// (about 140 KB) until the process exits. All calls share it, so calls that
// overlap on the GPU race on it; each call clears what must start at zero.
constexpr uint32_t kNoAllocMax = 1024;  // objects per allocation-free build (= kMediumMax)

struct NoAllocScratch {
    Rec rec[kNoAllocMax];
    Task medium[1];
    Task small[kNoAllocMax / 2 + 8];
    mgbvh_node nodes[2 * kNoAllocMax - 1];
    uint32_t lens[2 * kNoAllocMax - 1];
    uint8_t used[2 * kNoAllocMax];
    Counters ctr;
    uint32_t count;  // nodes written to the caller's array
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Counters to their initial state and every node slot of this build unused.
__global__ void noalloc_init_kernel(NoAllocScratch* S, uint32_t slots) {
    for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) S->used[i] = 0;
    uint32_t* c = reinterpret_cast<uint32_t*>(&S->ctr);
    for (uint32_t i = threadIdx.x; i < sizeof(Counters) / 4; i += blockDim.x) c[i] = 0;
    __syncthreads();
    if (threadIdx.x < 12) S->ctr.root_keys[threadIdx.x] = ((threadIdx.x % 6) < 3) ? kKeyPosInf : kKeyNegInf;
    if (threadIdx.x == 0) S->count = 0;
}

// Drops unused slots (leaves holding more than one object leave holes) and
// writes the nodes, with remapped child links, to the caller's array.
__global__ void __launch_bounds__(1024) noalloc_finish_kernel(NoAllocScratch* S, uint32_t slots,
                                                              mgbvh_node* out, uint32_t* out_lens,
                                                              uint32_t cap) {
    __shared__ uint32_t newidx[2 * kNoAllocMax];
    __shared__ uint32_t wsum[32];
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const uint32_t u0 = (2 * t < slots) ? S->used[2 * t] : 0u;
    const uint32_t u1 = (2 * t + 1 < slots) ? S->used[2 * t + 1] : 0u;
    const uint32_t v = u0 + u1;
    uint32_t inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t x = __shfl_up_sync(kFull, inc, d);
        if (lane >= static_cast<uint32_t>(d)) inc += x;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = wsum[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t x = __shfl_up_sync(kFull, w, d);
            if (lane >= static_cast<uint32_t>(d)) w += x;
        }
        wsum[lane] = w;  // inclusive
    }
    __syncthreads();
    const uint32_t excl = (warp ? wsum[warp - 1] : 0u) + inc - v;
    newidx[2 * t] = excl;
    newidx[2 * t + 1] = excl + u0;
    const uint32_t total = wsum[31];
    __syncthreads();
    if (t == 0) S->count = total;
    if (total > cap) {
        if (t == 0) set_error(&S->ctr, MGBVH_ERR_CAPACITY, kSiteCapacity);
        return;
    }
    for (uint32_t s = t; s < slots; s += blockDim.x) {
        if (!S->used[s]) continue;
        mgbvh_node nd = S->nodes[s];
        if (nd.child_node) nd.child_node = newidx[nd.child_node];
        out[newidx[s]] = nd;
        if (out_lens) out_lens[newidx[s]] = S->lens[s];
    }
}

}  // namespace mgbvh

// =================================================================== host

using namespace mgbvh;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct mgbvh_ctx {
    int device = 0;
    int sm_count = 148;
    uint32_t levels_hint = 0;
    uint32_t medium_max = kMediumMax;  // level-pass / subtree switch-over (speed only)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evp[3] = {nullptr, nullptr, nullptr};
    std::string err;
    DevBuf rec[2], tasks[2], bins[2], cbkeys[2], tile_task[2], tile_begin[2];
    DevBuf tile_hist, tile_lt, dec, medium, small, nodes, lens, used, newidx, widened, perm, ctr, cub_tmp;
    DevBuf bincode;  // per object of a level pass: its bin on each axis (5 bits each)
    DevBuf in_a, in_b, out_nodes, out_lens;
    DevBuf mesh_buf, toff_buf, noff_buf, mkeys;
    // forced medians of level-pass nodes: the waiting list, its working copy,
    // element offsets, per-node box keys, sort keys/values, flags and scan
    DevBuf med_list, med_work, med_off, med_seg, med_keys[2], med_vals[2], med_flag, med_scan;
    // persistent batched build (mgbvh_set_batch_mode): main queue entries, their
    // ready flags and centroid keys, small-queue ready flags, queue state
    bool batch_queue = false;
    DevBuf q, qready, qcb, qstate;
    void* h_qstate = nullptr;  // pinned QueueState of the last launch
    int queue_ctas[2] = {0, 0};  // resident CTAs of the 512- and 1024-record instances
    unsigned long long queue_wait_ns = 2000000000ull;
    uint32_t queue_hold = 0;
    uint32_t qcap = 0;  // main queue entries of the current batch
    // launch shapes (mgbvh_set_launch_shape; speed only): threads per CTA of
    // the warp-subtree kernel, persistent CTAs per SM (0: as many as fit)
    uint32_t small_threads = 256;
    uint32_t queue_per_sm = 0;
    // resident warps per SM of the warp-subtree kernel (mgbvh_set_small_occupancy)
    uint32_t small_warps = 24;
    void* pin = nullptr;  // pinned staging of a batch plan
    size_t pin_bytes = 0;
    bool graph_mode = false;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<unsigned char> graph_sig;
    uint32_t graph_levels = 0, graph_launches = 0;
    // learned split proposer (changes trees) and training-sample output;
    // learn_w points into learn_wt, the transposed copy of the parameters
    const void* learn_w = nullptr;
    DevBuf learn_wt, lref, rbins, tile_hist2;  // level-pass refine state (learned form)
    int learn_gate = 1;
    float learn_gate_thr = 0.0f;  // mgbvh_set_proposer_gate
    uint32_t learn_min_n = 0;
    float* learn_samples = nullptr;
    uint32_t learn_cap = 0;
    uint32_t* learn_count = nullptr;
    Counters* h_ctr = nullptr;
    Counters* h_init = nullptr;  // pinned, constant: the counters every build starts from
    // streamed output of host-pointer builds: the caller's page-locked node
    // and lens arrays receive slot chunks on cstream while the build runs
    cudaStream_t cstream = nullptr;
    cudaEvent_t evs[kStreamChunks] = {};
    DevBuf small2, medium2;  // subtrees of <= 32 objects and subtree CTA tasks sorted by slot chunk
    mgbvh_node* h_nodes_out = nullptr;
    uint32_t* h_lens_out = nullptr;
    bool streamed = false;  // the last build sent its node chunks on cstream
    uint32_t stream_slots = 0;  // > 0: this build streams (its node slot count)
};

namespace {

int fail(mgbvh_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return status;
}

#define MG_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(ctx, MGBVH_ERR_CUDA,                                               \
                        std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

int ensure(mgbvh_ctx* ctx, DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return MGBVH_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    const size_t want = bytes + bytes / 8;
    MG_CUDA(cudaMalloc(&b.p, want));
    b.bytes = want;
    return MGBVH_OK;
}

template <class T>
T* P_(DevBuf& b) {
    return reinterpret_cast<T*>(b.p);
}

struct Caps {
    uint32_t tasks, tiles, medium, small, nodes;
};

// List capacities for n objects over `meshes` roots, each a bound that no
// input can exceed: nodes above medium_max are disjoint at one level (<= n /
// (medium_max + 1) of them, spanning <= n / kTile + that many tiles); the
// queued subtrees of 33..medium_max objects are disjoint (none lies inside
// another), so there are <= n / 33 of them, however unbalanced the tree; the
// queued subtrees of 2..32 objects are disjoint too (<= n / 2).
Caps caps_for(uint32_t n, uint32_t medium_max, uint32_t meshes, uint32_t node_slots) {
    Caps c;
    c.tasks = n / (medium_max + 1) + 2;
    c.tiles = n / kTile + c.tasks + 2;
    c.medium = n / (kSmallMax + 1) + meshes + 8;
    c.small = n / 2 + meshes + 8;
    c.nodes = node_slots;
    return c;
}

int validate_settings(mgbvh_ctx* ctx, const mgbvh_settings* s) {
    if (!s) return fail(ctx, MGBVH_ERR_INVALID_ARG, "settings is NULL");
    if (s->min_leaf_objects < 1 || s->max_leaf_objects < 1)
        return fail(ctx, MGBVH_ERR_INVALID_ARG, "min/max leaf objects must be >= 1");
    if (s->min_leaf_objects > (1u << 30))
        return fail(ctx, MGBVH_ERR_INVALID_ARG, "min leaf objects too large");
    if (s->bins == 1 || s->bins > kMaxBins)
        return fail(ctx, MGBVH_ERR_UNSUPPORTED, "bins must be 0 (reference) or 2..32");
    if (s->adaptive_max_n > kSmallMax)
        return fail(ctx, MGBVH_ERR_UNSUPPORTED, "adaptive_max_n must be <= 32");
    if (s->adaptive_steps > 32)
        return fail(ctx, MGBVH_ERR_UNSUPPORTED, "adaptive_steps must be 0 (reference) or 1..32");
    return MGBVH_OK;
}

enum InputKind { kIndexed, kAabbs };

struct Input {
    InputKind kind;
    const float* verts;
    uint32_t stride_bytes;
    uint32_t nverts;
    const uint32_t* tris;
    const float* aabbs;
    uint32_t n;
};

const char* site_text(uint32_t site) {
    switch (site) {
        case kSiteIndex: return "a triangle index is past the vertex count";
        case kSiteCount: return "partition count differs from the split's count (bvh/src/lib.rs:621-634)";
        case kSiteContain: return "a centroid lies outside its child's bounds (bvh/src/lib.rs:637-646)";
        case kSiteMedian: return "forced median: a half's count differs from len / 2 (bvh/src/lib.rs:621-634)";
        case kSiteCapacity: return "internal task list overflow";
        case kSiteMeshIndex: return "an instance names a mesh past mesh_count";
        default: return "device error";
    }
}

#ifndef MGBVH_PDL
#define MGBVH_PDL 1  // 1: pipeline kernels launched with programmatic stream serialization
#endif

// Launches a pipeline kernel on stream `st`. With MGBVH_PDL the launch
// allows programmatic stream serialization: the kernel's CTAs may be
// scheduled while the previous kernel in the stream finishes, and wait in
// pdl_enter() (griddepcontrol.wait) until it has completed, so the launch
// latency between dependent kernels overlaps the previous kernel's tail.
template <typename... KArgs, typename... Args>
void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = MGBVH_PDL ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);  // errors surface at cudaGetLastError
}

// Level passes (nodes above medium_max), then the medium and small subtree
// kernels, on the context's stream. Root tasks are already queued.
// fixed_levels > 0: launch exactly that many level passes and never read
// back (the form a CUDA graph captures); 0: read the next level's count at
// the end of each batch of levels.
// optimistic (single builds with a level-count hint from an earlier build):
// launch exactly the hinted number of levels and go on to the subtree
// kernels without a host read in between; the caller checks afterwards that
// no task was left for a further level (and rebuilds if one was).
int run_pipeline(mgbvh_ctx* ctx, const Caps& C, const Params& P, const Out& O, Rec* rec0, Rec* rec1,
                 bool has_large, uint32_t fixed_levels, uint32_t& launches, uint32_t& levels,
                 bool optimistic = false) {
    const cudaStream_t sm = ctx->stream;
    Counters* d_ctr = O.ctr;
    // Level passes over the large nodes. Kernels read their task and tile
    // counts on the device, so levels are launched in batches and the host
    // reads the next level's count only at the end of a batch.
    const int tile_grid = (int)std::min<uint32_t>(C.tiles, (uint32_t)ctx->sm_count * 8u);
    const int eval_grid = (int)std::min<uint32_t>((C.tasks + 3) / 4, (uint32_t)ctx->sm_count * 4u);
    uint32_t level = 0;
    bool more = has_large;
    if (!fixed_levels) ctx->h_ctr->error = 0;
    Learn LN;
    LN.w = static_cast<const __nv_bfloat16*>(ctx->learn_w);
    LN.gate = ctx->learn_gate;
    LN.gate_thr = ctx->learn_gate_thr;
    LN.min_n = ctx->learn_min_n;
    LN.samples = ctx->learn_samples;
    LN.cap = ctx->learn_cap;
    LN.count = ctx->learn_count;
    bool first_batch = true;
    while (more) {
        const uint32_t batch = fixed_levels ? fixed_levels
                                            : (optimistic ? ctx->levels_hint
                                                          : (first_batch ? std::max(ctx->levels_hint, 4u) : 2u));
        first_batch = false;
        for (uint32_t bl = 0; bl < batch; ++bl, ++level) {
            // buffers alternate between two sets; level counters rotate over three slots
            const uint32_t bf = level & 1u, nx = bf ^ 1u, lv = level % 3u;
            launches += 3;
            EvalArgs A;
            A.tasks = P_<Task>(ctx->tasks[bf]);
            A.lv = lv;
            A.bins = P_<uint32_t>(ctx->bins[bf]);
            A.cbkeys = P_<uint32_t>(ctx->cbkeys[bf]);
            A.tile_hist = P_<uint32_t>(ctx->tile_hist);
            A.tile_lt = P_<uint32_t>(ctx->tile_lt);
            A.dec = P_<Decision>(ctx->dec);
            A.next_tasks = P_<Task>(ctx->tasks[nx]);
            A.next_bins = P_<uint32_t>(ctx->bins[nx]);
            A.next_cbkeys = P_<uint32_t>(ctx->cbkeys[nx]);
            A.next_tile_task = P_<uint32_t>(ctx->tile_task[nx]);
            A.next_tile_begin = P_<uint32_t>(ctx->tile_begin[nx]);
            A.medium = P_<Task>(ctx->medium);
            A.small = P_<Task>(ctx->small);
            A.cap_tasks = C.tasks;
            A.cap_tiles = C.tiles;
            A.cap_medium = C.medium;
            A.cap_small = C.small;
            A.lw = LN.w;
            A.lgate = LN.gate;
            A.lgate_thr = LN.gate_thr;
            A.lmin_n = LN.min_n;
            A.refine = LN.w ? P_<LvlRefine>(ctx->lref) : nullptr;
            A.rbins = LN.w ? P_<uint32_t>(ctx->rbins) : nullptr;
            A.tile_hist2 = LN.w ? P_<uint32_t>(ctx->tile_hist2) : nullptr;
            A.med = P_<Task>(ctx->med_list);
            launch_k(lvl_bin_kernel, tile_grid, kTileThreads, 0, sm,
                P_<Task>(ctx->tasks[bf]), P_<uint32_t>(ctx->cbkeys[bf]), P_<uint32_t>(ctx->bins[bf]),
                P_<uint32_t>(ctx->tile_task[bf]), P_<uint32_t>(ctx->tile_begin[bf]),
                P_<uint32_t>(ctx->tile_hist), C.tiles, rec0, rec1, P_<uint16_t>(ctx->bincode), d_ctr, lv, P);
            launch_k(LN.w ? lvl_eval_kernel<true> : lvl_eval_kernel<false>, eval_grid, 128, LN.w ? kEvalWeightBytes : 0,
                     sm, A, P, O);
            if (LN.samples) {
                launch_k(lvl_sample_kernel, ctx->sm_count * 2, 256, 0, sm,
                    A.tasks, A.dec, A.bins, A.cbkeys, rec0, rec1, d_ctr, lv, P, LN);
                launches++;
            }
            if (LN.w) {
                launch_k(lvl_refine_bin_kernel, tile_grid, kTileThreads, 0, sm,
                    A.tasks, A.cbkeys, A.refine, A.rbins, P_<uint32_t>(ctx->tile_task[bf]),
                    P_<uint32_t>(ctx->tile_begin[bf]), P_<uint32_t>(ctx->tile_hist2),
                    P_<uint32_t>(ctx->tile_hist), C.tiles, rec0, rec1, P_<uint16_t>(ctx->bincode), d_ctr, lv);
                launch_k(lvl_eval2_kernel, eval_grid, 128, 0, sm, A, P, O);
                launches += 2;
            }
            launch_k(lvl_part_kernel, tile_grid, kTileThreads, 0, sm,
                P_<Task>(ctx->tasks[bf]), P_<Decision>(ctx->dec), P_<uint32_t>(ctx->tile_task[bf]),
                P_<uint32_t>(ctx->tile_begin[bf]), P_<uint32_t>(ctx->tile_lt), rec0, rec1,
                P_<uint16_t>(ctx->bincode), P_<uint32_t>(ctx->cbkeys[nx]), lv, O);
        }
        MG_CUDA(cudaGetLastError());
        if (fixed_levels || optimistic) break;
        MG_CUDA(cudaMemcpyAsync(ctx->h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
        if (ctx->h_ctr->error) break;
        more = ctx->h_ctr->lvl[level % 3u][0] > 0;
    }
    if (has_large) {
        if (!fixed_levels && !optimistic) ctx->levels_hint = level;
        levels = level;
    }
    if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->evp[1], sm));
    if (fixed_levels || !ctx->h_ctr->error) {
        // medium subtrees: count read on the device
        const uint32_t mgrid = std::min<uint32_t>(C.medium, (uint32_t)ctx->sm_count * 4u);
        // subtrees hold at most P.medium_max objects: the smaller-capacity
        // instance leaves room for more CTAs per SM
        // the learned instance only where a subtree node can reach the
        // network's size gate (or samples are collected)
        const bool lrn = (LN.w && LN.min_n <= P.medium_max) || LN.samples,
                   small_cap = P.medium_max <= kMediumSmallCap;
        const uint32_t mgrid_s =
            std::min<uint32_t>(C.medium, (uint32_t)ctx->sm_count * (uint32_t)MGBVH_MEDIUM_SMALL_CTAS);
        auto medium = [&](const Task* tasks, const uint32_t* range) {
            if (lrn && small_cap)
                launch_k(medium_kernel<true, kMediumSmallCap>, mgrid_s, kMediumThreads, medium_smem_bytes<true, kMediumSmallCap>(), sm,
                    tasks, rec0, rec1, P_<Task>(ctx->small), C.small, P, O, LN, range);
            else if (lrn)
                launch_k(medium_kernel<true, kMediumMax>, mgrid, kMediumThreads, medium_smem_bytes<true, kMediumMax>(), sm,
                    tasks, rec0, rec1, P_<Task>(ctx->small), C.small, P, O, LN, range);
            else if (small_cap)
                launch_k(medium_kernel<false, kMediumSmallCap>, mgrid_s, kMediumThreads, medium_smem_bytes<false, kMediumSmallCap>(), sm,
                    tasks, rec0, rec1, P_<Task>(ctx->small), C.small, P, O, LN, range);
            else
                launch_k(medium_kernel<false, kMediumMax>, mgrid, kMediumThreads, medium_smem_bytes<false, kMediumMax>(), sm,
                    tasks, rec0, rec1, P_<Task>(ctx->small), C.small, P, O, LN, range);
        };
        // small subtrees: count read on the device; grid sized for full occupancy
        const bool lv_small = P.adaptive_steps == 0 && P.adaptive_max_n == kSmallMax;
        auto small = ctx->small_warps == 16u ? (lv_small ? small_kernel<true, 2> : small_kernel<false, 2>)
                                             : (lv_small ? small_kernel<true, 3> : small_kernel<false, 3>);
        // as many warps as 8 CTAs of 256 threads per SM, whatever the CTA size
        const int small_grid = ctx->sm_count * (2048 / (int)ctx->small_threads);
        if (ctx->stream_slots && ctx->h_nodes_out) {
            // streamed output: the subtrees of both kinds run chunk by chunk
            // of node slots (the chunk of their children pair): chunk c's
            // subtree CTAs, then the subtrees of <= 32 objects of chunk c
            // (all queued by then: a subtree's children pairs come after its
            // own). After them no later launch changes chunk c's slots (the
            // roots of later subtrees, which may lie anywhere before, hold
            // their final words already), so the chunk goes to the host on
            // the copy stream while the next chunks run.
            const uint32_t S = ctx->stream_slots;
            if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->evp[2], sm));
            launch_k(medium_count_kernel, ctx->sm_count * 2, 256, 0, sm, P_<Task>(ctx->medium), O, S);
            launch_k(medium_sort_kernel, ctx->sm_count * 2, 256, 0, sm, P_<Task>(ctx->medium), P_<Task>(ctx->medium2),
                                                                   d_ctr, S);
            launches += 2;
            for (uint32_t c = 0; c < kStreamChunks; ++c) {
                medium(P_<Task>(ctx->medium2), d_ctr->mrange + c);
                launch_k(small_select_kernel, ctx->sm_count, 256, 0, sm, P_<Task>(ctx->small), P_<Task>(ctx->small2),
                                                                   C.small, O, c, S);
                launch_k(small, small_grid, ctx->small_threads, 0, sm, P_<Task>(ctx->small2), rec0, rec1, P, O,
                                                         d_ctr->srange + c);
                launches += 3;
                MG_CUDA(cudaEventRecord(ctx->evs[c], sm));
                MG_CUDA(cudaStreamWaitEvent(ctx->cstream, ctx->evs[c], 0));
                const uint32_t r0 = stream_chunk_begin(c, S), r1 = stream_chunk_begin(c + 1, S);
                if (r1 <= r0) continue;
                MG_CUDA(cudaMemcpyAsync(ctx->h_nodes_out + r0, O.nodes + r0, sizeof(mgbvh_node) * (size_t)(r1 - r0),
                                        cudaMemcpyDeviceToHost, ctx->cstream));
                if (ctx->h_lens_out)
                    MG_CUDA(cudaMemcpyAsync(ctx->h_lens_out + r0, O.lens + r0, 4ull * (r1 - r0),
                                            cudaMemcpyDeviceToHost, ctx->cstream));
            }
            ctx->streamed = true;
        } else {
            medium(P_<Task>(ctx->medium), nullptr);
            launches++;
            if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->evp[2], sm));
            launch_k(small, small_grid, ctx->small_threads, 0, sm, P_<Task>(ctx->small), rec0, rec1, P, O, nullptr);
            launches++;
        }
        MG_CUDA(cudaGetLastError());
    } else {
        MG_CUDA(cudaEventRecord(ctx->evp[2], sm));
    }
    return MGBVH_OK;
}

// Forced medians of level-pass nodes (the median kernels above). The nodes
// that lvl_eval_kernel queued during the pipeline are split here, then their
// subtrees are built by another pipeline run, which may queue further nodes;
// until none is left. The waiting subtrees are disjoint from everything the
// pipeline built, and their node slots follow from the closed-form numbering,
// so building them afterwards gives the same tree. The counters in
// ctx->h_ctr are current on entry (the caller synchronized the stream) and on
// return.
int run_medians(mgbvh_ctx* ctx, const Caps& C, const Params& P, const Out& O, Rec* rec0, Rec* rec1,
                uint32_t n_objects, uint32_t& launches) {
    const cudaStream_t sm = ctx->stream;
    Counters* d_ctr = O.ctr;
    // chunks streamed to the host during the pipeline miss the waiting
    // subtrees: let them land, then the caller copies the whole array
    if (ctx->streamed) {
        MG_CUDA(cudaStreamSynchronize(ctx->cstream));
        ctx->streamed = false;
    }
    struct Restore {  // the level-count hint and streaming belong to the main pipeline run
        mgbvh_ctx* c;
        uint32_t hint, slots;
        ~Restore() {
            c->levels_hint = hint;
            c->stream_slots = slots;
        }
    } restore{ctx, ctx->levels_hint, ctx->stream_slots};
    ctx->stream_slots = 0;
    const int grid = ctx->sm_count * 8;
    int rc;
    while (!ctx->h_ctr->error && ctx->h_ctr->n_med) {
        const uint32_t np = ctx->h_ctr->n_med;
        if (np > C.tasks) return fail(ctx, MGBVH_ERR_CAPACITY, "internal task list overflow");
        std::vector<Task> ht(np);
        MG_CUDA(cudaMemcpyAsync(ht.data(), ctx->med_list.p, sizeof(Task) * np, cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
        std::vector<uint32_t> off(np + 1);
        uint64_t E = 0;
        for (uint32_t i = 0; i < np; ++i) {
            off[i] = static_cast<uint32_t>(E);
            E += ht[i].len;
        }
        if (E > n_objects) return fail(ctx, MGBVH_ERR_ASSERT, "forced median: waiting nodes overlap");
        off[np] = static_cast<uint32_t>(E);
        if ((rc = ensure(ctx, ctx->med_work, sizeof(Task) * np)) != MGBVH_OK) return rc;
        if ((rc = ensure(ctx, ctx->med_off, 4ull * (np + 1))) != MGBVH_OK) return rc;
        if ((rc = ensure(ctx, ctx->med_seg, sizeof(MedSeg) * np)) != MGBVH_OK) return rc;
        for (int i = 0; i < 2; ++i) {
            if ((rc = ensure(ctx, ctx->med_keys[i], 8 * E)) != MGBVH_OK) return rc;
            if ((rc = ensure(ctx, ctx->med_vals[i], 4 * E)) != MGBVH_OK) return rc;
        }
        if ((rc = ensure(ctx, ctx->med_flag, 4 * E)) != MGBVH_OK) return rc;
        if ((rc = ensure(ctx, ctx->med_scan, 4 * E)) != MGBVH_OK) return rc;
        const Task* mt = P_<Task>(ctx->med_work);
        const uint32_t* moff = P_<uint32_t>(ctx->med_off);
        MedSeg* seg = P_<MedSeg>(ctx->med_seg);
        unsigned long long* k0 = P_<unsigned long long>(ctx->med_keys[0]);
        unsigned long long* k1 = P_<unsigned long long>(ctx->med_keys[1]);
        uint32_t* v0 = P_<uint32_t>(ctx->med_vals[0]);
        uint32_t* v1 = P_<uint32_t>(ctx->med_vals[1]);
        uint32_t* flag = P_<uint32_t>(ctx->med_flag);
        uint32_t* scan = P_<uint32_t>(ctx->med_scan);
        const uint32_t e32 = static_cast<uint32_t>(E);
        MG_CUDA(cudaMemcpyAsync(ctx->med_off.p, off.data(), 4ull * (np + 1), cudaMemcpyHostToDevice, sm));
        MG_CUDA(cudaMemcpyAsync(ctx->med_work.p, ctx->med_list.p, sizeof(Task) * np, cudaMemcpyDeviceToDevice, sm));
        med_reset_kernel<<<1, 32, 0, sm>>>(d_ctr);
        med_init_kernel<<<std::min<uint32_t>((np * 48u + 255u) / 256u, 1024u), 256, 0, sm>>>(seg, np);
        const int end_bit = 32 + (np > 1 ? 32 - __builtin_clz(np - 1) : 0);
        const int eg = (int)std::min<uint64_t>((E + 255) / 256, (uint64_t)grid);
        for (uint32_t axis = 0; axis < 3; ++axis) {
            med_key_kernel<<<eg, 256, 0, sm>>>(mt, moff, np, e32, rec0, rec1, axis, k0, v0);
            size_t tb = 0, ts = 0;
            MG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, v0, v1, (int)e32, 0, end_bit, sm));
            MG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, ts, flag, scan, (int)e32, sm));
            if ((rc = ensure(ctx, ctx->cub_tmp, std::max(tb, ts))) != MGBVH_OK) return rc;
            tb = ts = ctx->cub_tmp.bytes;
            MG_CUDA(cub::DeviceRadixSort::SortPairs(ctx->cub_tmp.p, tb, k0, k1, v0, v1, (int)e32, 0, end_bit, sm));
            med_flag_kernel<<<eg, 256, 0, sm>>>(mt, moff, np, e32, k0, k1, v1, flag);
            MG_CUDA(cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, ts, flag, scan, (int)e32, sm));
            med_scatter_kernel<<<eg, 256, 0, sm>>>(mt, moff, np, e32, rec0, rec1, axis, flag, scan, seg, P, O);
            launches += 5;
        }
        MedOut M;
        M.tasks = P_<Task>(ctx->tasks[0]);
        M.bins = P_<uint32_t>(ctx->bins[0]);
        M.cbkeys = P_<uint32_t>(ctx->cbkeys[0]);
        M.tile_task = P_<uint32_t>(ctx->tile_task[0]);
        M.tile_begin = P_<uint32_t>(ctx->tile_begin[0]);
        M.medium = P_<Task>(ctx->medium);
        M.small = P_<Task>(ctx->small);
        M.cap_tasks = C.tasks;
        M.cap_tiles = C.tiles;
        M.cap_medium = C.medium;
        M.cap_small = C.small;
        med_finish_kernel<<<std::min<uint32_t>((np + 3) / 4, 1024u), 128, 0, sm>>>(mt, np, seg, M, P, O);
        launches += 3;
        MG_CUDA(cudaGetLastError());
        MG_CUDA(cudaMemcpyAsync(ctx->h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
        if (ctx->h_ctr->error) break;
        uint32_t levels = 0;
        if ((rc = run_pipeline(ctx, C, P, O, rec0, rec1, ctx->h_ctr->lvl[0][0] > 0, 0, launches, levels)) !=
            MGBVH_OK)
            return rc;
        MG_CUDA(cudaMemcpyAsync(ctx->h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
    }
    return MGBVH_OK;
}

// Runs a build whose inputs are device-resident. Outputs go to device memory:
// d_nodes (capacity cap), d_lens (nullable), d_perm. Returns status.
int run_build(mgbvh_ctx* ctx, const Input& in, const mgbvh_settings* st, mgbvh_node* d_nodes,
              uint32_t cap, uint32_t* d_lens, uint32_t* d_perm, uint32_t* out_count,
              mgbvh_stats* stats) {
    const uint32_t n = in.n;
    const cudaStream_t sm = ctx->stream;
    if (n > 0x7FFFFFFFu) return fail(ctx, MGBVH_ERR_UNSUPPORTED, "more than 2^31-1 objects");
    const Caps C = caps_for(n, ctx->medium_max, 1, 2 * n - 1);
    int rc;
#define ENS(buf, bytes) \
    if ((rc = ensure(ctx, buf, (bytes))) != MGBVH_OK) return rc
    ENS(ctx->rec[0], sizeof(Rec) * (size_t)n);
    ENS(ctx->rec[1], sizeof(Rec) * (size_t)n);
    for (int i = 0; i < 2; ++i) {
        ENS(ctx->tasks[i], sizeof(Task) * (size_t)C.tasks);
        ENS(ctx->bins[i], 4ull * kBinWords * C.tasks);
        ENS(ctx->cbkeys[i], 24ull * C.tasks);
        ENS(ctx->tile_task[i], 4ull * C.tiles);
        ENS(ctx->tile_begin[i], 4ull * C.tiles);
    }
    ENS(ctx->tile_hist, 4ull * 96 * C.tiles);  // [axis][bin][tile]
    ENS(ctx->tile_lt, 4ull * C.tiles);
    ENS(ctx->bincode, 2ull * n);
    ENS(ctx->dec, sizeof(Decision) * (size_t)C.tasks);
    ENS(ctx->med_list, sizeof(Task) * (size_t)C.tasks);
    ENS(ctx->medium, sizeof(Task) * (size_t)C.medium);
    ENS(ctx->small, sizeof(Task) * (size_t)C.small);
    ENS(ctx->nodes, sizeof(mgbvh_node) * (size_t)C.nodes);
    ENS(ctx->lens, 4ull * C.nodes);
    ENS(ctx->used, (size_t)C.nodes);
    ENS(ctx->ctr, sizeof(Counters));
    if (ctx->learn_w) {
        ENS(ctx->lref, sizeof(LvlRefine) * (size_t)C.tasks);
        ENS(ctx->rbins, 4ull * kRBinWords * C.tasks);
        ENS(ctx->tile_hist2, 4ull * 34 * C.tiles);  // [proposal * 17 + interval][tile]
    }
#undef ENS
    Params P;
    P.min_leaf = st->min_leaf_objects;
    P.max_leaf = st->max_leaf_objects;
    P.max_depth = st->max_depth;
    P.bins = st->bins;
    P.adaptive_max_n = st->adaptive_max_n;
    P.adaptive_steps = st->adaptive_steps;
    P.medium_max = ctx->medium_max;

    Counters* d_ctr = P_<Counters>(ctx->ctr);
    // from pinned memory: an asynchronous copy (a pageable source would stall the host)
    MG_CUDA(cudaMemcpyAsync(d_ctr, ctx->h_init, sizeof(Counters), cudaMemcpyHostToDevice, sm));
    MG_CUDA(cudaMemsetAsync(ctx->used.p, 0, (size_t)C.nodes, sm));

    Out O;
    // with room for every slot, nodes (and lens) go straight to the caller's
    // buffers; scratch copies are made only when holes must be compacted
    const bool direct = cap >= C.nodes;
    O.nodes = direct ? d_nodes : P_<mgbvh_node>(ctx->nodes);
    O.lens = (direct && d_lens) ? d_lens : P_<uint32_t>(ctx->lens);
    O.used = P_<uint8_t>(ctx->used);
    O.perm = d_perm;
    O.ctr = d_ctr;
    O.node_cap = C.nodes;
    Rec* rec0 = P_<Rec>(ctx->rec[0]);
    Rec* rec1 = P_<Rec>(ctx->rec[1]);

    MG_CUDA(cudaEventRecord(ctx->ev0, sm));
    const int prep_blocks = (int)std::min<uint32_t>((n + 255) / 256, 148u * 8u);
    if (in.kind == kIndexed)
        launch_k(prep_indexed_kernel, prep_blocks, 256, 0, sm, in.verts, in.stride_bytes / 4, in.nverts,
                                                          in.tris, n, rec0, d_ctr);
    else
        launch_k(prep_aabbs_kernel, prep_blocks, 256, 0, sm, in.aabbs, n, rec0, d_ctr);

    const bool root_leaf = n <= 1 || st->max_depth == 0 ||
                           (n <= st->max_leaf_objects && n < 2u * st->min_leaf_objects);
    const uint32_t cls = root_leaf ? 0u : (n <= kSmallMax ? 1u : (n <= P.medium_max ? 2u : 3u));
    // streamed output (host-pointer builds into page-locked arrays): with one
    // object per leaf every subtree of <= 32 objects splits at its root, whose
    // words are then known before the small kernel runs
    ctx->stream_slots = 0;
    if (ctx->h_nodes_out && direct && st->max_leaf_objects == 1 && cls >= 2) {
        if ((rc = ensure(ctx, ctx->small2, sizeof(Task) * (size_t)C.small)) != MGBVH_OK) return rc;
        if ((rc = ensure(ctx, ctx->medium2, sizeof(Task) * (size_t)C.medium)) != MGBVH_OK) return rc;
        ctx->stream_slots = C.nodes;
    }
    const uint32_t ntiles0 = (n + kTile - 1) / kTile;
    const float* bb = st->bounds;
    {
        const int blocks = (int)std::min<uint32_t>((std::max(n, ntiles0) + 255) / 256 + 1, 1024u);
        launch_k(init_root_kernel, blocks, 256, 0, sm,
            n, cls, st->has_bounds, bb[0], bb[1], bb[2], bb[3], bb[4], bb[5], P_<Task>(ctx->tasks[0]),
            P_<uint32_t>(ctx->bins[0]), P_<uint32_t>(ctx->cbkeys[0]), P_<uint32_t>(ctx->tile_task[0]),
            P_<uint32_t>(ctx->tile_begin[0]), P_<Task>(ctx->medium), P_<Task>(ctx->small), O, ntiles0,
            st->max_depth);
    }
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaEventRecord(ctx->evp[0], sm));
    uint32_t launches = 2, levels = 0;
    (void)ntiles0;

    const bool optimistic = cls == 3 && ctx->levels_hint > 0;
    if ((rc = run_pipeline(ctx, C, P, O, rec0, rec1, cls == 3, 0, launches, levels, optimistic)) != MGBVH_OK)
        return rc;
    MG_CUDA(cudaEventRecord(ctx->ev1, sm));
    MG_CUDA(cudaMemcpyAsync(ctx->h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, sm));
    MG_CUDA(cudaStreamSynchronize(sm));
    if (optimistic && ctx->h_ctr->lvl[levels % 3u][0] != 0) {
        // the tree needs more level passes than the hint: build again, reading
        // the task count after every batch of levels
        ctx->levels_hint = 0;
        return run_build(ctx, in, st, d_nodes, cap, d_lens, d_perm, out_count, stats);
    }
    if (!ctx->h_ctr->error && ctx->h_ctr->n_med) {
        // level-pass nodes that need the forced median
        if ((rc = run_medians(ctx, C, P, O, rec0, rec1, n, launches)) != MGBVH_OK) return rc;
        MG_CUDA(cudaEventRecord(ctx->ev1, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
    }
    const Counters hc = *ctx->h_ctr;
    if (hc.error) {
        return fail(ctx, (int)hc.error, site_text(hc.error_site));
    }
    float ms = 0.0f;
    MG_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));

    // node count and compaction
    uint32_t count = C.nodes;
    if (hc.holes > 0) {
        if (direct) {  // the compaction reads the slots from scratch
            MG_CUDA(cudaMemcpyAsync(ctx->nodes.p, d_nodes, sizeof(mgbvh_node) * (size_t)C.nodes,
                                    cudaMemcpyDeviceToDevice, sm));
            if (d_lens)
                MG_CUDA(cudaMemcpyAsync(ctx->lens.p, d_lens, 4ull * C.nodes, cudaMemcpyDeviceToDevice, sm));
        }
        if ((rc = ensure(ctx, ctx->newidx, 4ull * C.nodes)) != MGBVH_OK) return rc;
        if ((rc = ensure(ctx, ctx->widened, 4ull * C.nodes)) != MGBVH_OK) return rc;
        widen_used_kernel<<<std::min<uint32_t>((C.nodes + 255) / 256, 4096u), 256, 0, sm>>>(
            P_<uint8_t>(ctx->used), C.nodes, P_<uint32_t>(ctx->widened));
        size_t tmp = 0;
        MG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, P_<uint32_t>(ctx->widened),
                                              P_<uint32_t>(ctx->newidx), C.nodes, sm));
        if ((rc = ensure(ctx, ctx->cub_tmp, tmp)) != MGBVH_OK) return rc;
        MG_CUDA(cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, tmp, P_<uint32_t>(ctx->widened),
                                              P_<uint32_t>(ctx->newidx), C.nodes, sm));
        uint32_t last_idx = 0;
        uint8_t last_used = 0;
        MG_CUDA(cudaMemcpyAsync(&last_idx, P_<uint32_t>(ctx->newidx) + (C.nodes - 1), 4,
                                cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaMemcpyAsync(&last_used, P_<uint8_t>(ctx->used) + (C.nodes - 1), 1,
                                cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
        count = last_idx + last_used;
        if (count > cap) return fail(ctx, MGBVH_ERR_CAPACITY, "node_capacity is smaller than the tree");
        compact_kernel<<<std::min<uint32_t>((C.nodes + 255) / 256, 4096u), 256, 0, sm>>>(
            P_<mgbvh_node>(ctx->nodes), P_<uint32_t>(ctx->lens), P_<uint8_t>(ctx->used),
            P_<uint32_t>(ctx->newidx), C.nodes, d_nodes, d_lens);
        MG_CUDA(cudaGetLastError());
        launches += 2;
    } else if (!direct) {
        if (count > cap) return fail(ctx, MGBVH_ERR_CAPACITY, "node_capacity is smaller than the tree");
        MG_CUDA(cudaMemcpyAsync(d_nodes, ctx->nodes.p, sizeof(mgbvh_node) * (size_t)count,
                                cudaMemcpyDeviceToDevice, sm));
        if (d_lens)
            MG_CUDA(cudaMemcpyAsync(d_lens, ctx->lens.p, 4ull * count, cudaMemcpyDeviceToDevice, sm));
    }
    if (hc.holes > 0 || !direct) MG_CUDA(cudaStreamSynchronize(sm));
    *out_count = count;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->construction_time = ms * 1e-3;
        stats->node_count = count;
        stats->total_object_count = n;
        stats->height = hc.height;
        stats->max_depth = st->max_depth;
        stats->median_splits = hc.median_splits;
        stats->learned_splits = hc.learned;
        stats->depth_capped_leaves = hc.depth_capped;
        stats->kernel_launches = launches;
        stats->levels = levels;
        float pm[4] = {0.f, 0.f, 0.f, 0.f};
        cudaEventElapsedTime(&pm[0], ctx->ev0, ctx->evp[0]);
        cudaEventElapsedTime(&pm[1], ctx->evp[0], ctx->evp[1]);
        cudaEventElapsedTime(&pm[2], ctx->evp[1], ctx->evp[2]);
        cudaEventElapsedTime(&pm[3], ctx->evp[2], ctx->ev1);
        for (int i = 0; i < 4; ++i) stats->phase_seconds[i] = pm[i] * 1e-3;
        const uint32_t MINs = st->min_leaf_objects, MAXs = st->max_leaf_objects;
        stats->feasible = (MINs == MAXs) ? (n % MINs == 0) : (MAXs >= 2 * MINs - 1);
        if (st->profiling_info) {
            // leaf statistics as bvh/src/lib.rs:769-788 computes them
            std::vector<mgbvh_node> hn(count);
            std::vector<uint32_t> hl(count);
            MG_CUDA(cudaMemcpy(hn.data(), d_nodes, sizeof(mgbvh_node) * (size_t)count,
                               cudaMemcpyDeviceToHost));
            const uint32_t* lens_src = d_lens ? d_lens : nullptr;
            if (lens_src) {
                MG_CUDA(cudaMemcpy(hl.data(), lens_src, 4ull * count, cudaMemcpyDeviceToHost));
            } else if (hc.holes == 0) {
                MG_CUDA(cudaMemcpy(hl.data(), ctx->lens.p, 4ull * count, cudaMemcpyDeviceToHost));
            } else {
                // compacted lens were not requested: compact again into scratch
                if ((rc = ensure(ctx, ctx->out_lens, 4ull * count)) != MGBVH_OK) return rc;
                if ((rc = ensure(ctx, ctx->out_nodes, sizeof(mgbvh_node) * (size_t)count)) != MGBVH_OK)
                    return rc;
                compact_kernel<<<std::min<uint32_t>((C.nodes + 255) / 256, 4096u), 256, 0, sm>>>(
                    P_<mgbvh_node>(ctx->nodes), P_<uint32_t>(ctx->lens), P_<uint8_t>(ctx->used),
                    P_<uint32_t>(ctx->newidx), C.nodes, P_<mgbvh_node>(ctx->out_nodes),
                    P_<uint32_t>(ctx->out_lens));
                MG_CUDA(cudaStreamSynchronize(sm));
                MG_CUDA(cudaMemcpy(hl.data(), ctx->out_lens.p, 4ull * count, cudaMemcpyDeviceToHost));
            }
            std::vector<uint32_t> leaf;
            for (uint32_t i = 1; i < count; ++i)
                if (hn[i].child_node == 0) leaf.push_back(hl[i]);
            stats->leaf_node_count = (uint32_t)leaf.size();
            stats->min_leaf_object_count = leaf.empty() ? n : *std::min_element(leaf.begin(), leaf.end());
            stats->max_leaf_object_count = leaf.empty() ? n : *std::max_element(leaf.begin(), leaf.end());
            uint32_t sum = 0;
            for (uint32_t l : leaf) sum += l;
            const double avg = (double)sum / (double)leaf.size();
            double var = 0.0;
            for (uint32_t l : leaf) var += ((double)l - avg) * ((double)l - avg);
            stats->avg_leaf_object_count = avg;
            stats->stddev_leaf_object_count = std::sqrt(var / (double)leaf.size());
        }
    }
    const uint32_t MIN = st->min_leaf_objects, MAX = st->max_leaf_objects;
    const bool feasible = (MIN == MAX) ? (n % MIN == 0) : (MAX >= 2 * MIN - 1);  // :710-714
    return feasible ? MGBVH_OK : MGBVH_WARN_INFEASIBLE;
}


// Batched build over several meshes (see include/mgbvh.h).
//
// Plan (host): object and node offsets of every mesh, each root's list and
// tiles. Device work (enqueue_batch): inputs of the plan copied from pinned
// staging, record prep, roots, the pipeline, and either a read-back per
// batch of levels (eager) or a fixed number of levels and the copy of the
// results to the caller (graph capture). With graph capture on, the first
// build of a mesh set runs eagerly and learns its level count; later builds
// of the same set (same pointers, counts and settings) replay one CUDA graph
// of the whole batch with one spare level, and fall back to the eager path
// if the spare level turns out to have work (a deeper tree).
struct BatchPlan {
    uint32_t nm = 0, n = 0, slots = 0, n_large = 0, n_medium = 0, n_small = 0, tiles = 0;
    std::vector<DevMesh> hm;
    std::vector<uint32_t> toffs, noffs;
};

int plan_batch(mgbvh_ctx* ctx, const mgbvh_mesh_desc* meshes, uint32_t nm, const mgbvh_settings* st,
               BatchPlan& B) {
    B.nm = nm;
    B.hm.assign(nm, DevMesh());
    B.toffs.assign(nm + 1, 0);
    B.noffs.assign(nm + 1, 0);
    uint64_t total = 0, slots = 0;
    for (uint32_t m = 0; m < nm; ++m) {
        const mgbvh_mesh_desc& d = meshes[m];
        DevMesh& M = B.hm[m];
        std::memset(&M, 0, sizeof(M));
        const bool tri = d.vertices != nullptr;
        if (d.count && tri && (!d.triangles || d.vertex_stride_bytes < 12 || d.vertex_stride_bytes % 4))
            return fail(ctx, MGBVH_ERR_INVALID_ARG, "mesh " + std::to_string(m) + ": bad vertex data");
        if (d.count && !tri && !d.aabbs)
            return fail(ctx, MGBVH_ERR_INVALID_ARG, "mesh " + std::to_string(m) + ": no objects");
        M.verts = d.vertices;
        M.tris = d.triangles;
        M.aabbs = d.aabbs;
        M.stride_floats = d.vertex_stride_bytes / 4;
        M.nverts = d.vertex_count;
        M.n = d.count;
        M.tbase = (uint32_t)total;
        M.nbase = (uint32_t)slots;
        M.has_bounds = d.has_bounds;
        for (int i = 0; i < 6; ++i) M.bounds[i] = d.bounds[i];
        B.toffs[m] = (uint32_t)total;
        B.noffs[m] = (uint32_t)slots;
        total += d.count;
        slots += d.count ? 2ull * d.count - 1 : 0;
        if (total > 0x7FFFFFFFull || slots > 0xFFFFFFFEull)
            return fail(ctx, MGBVH_ERR_UNSUPPORTED, "batch above 2^31-1 objects");
        const uint32_t n = d.count;
        if (n == 0) {
            M.cls = 4;
            continue;
        }
        const bool leaf = n <= 1 || st->max_depth == 0 ||
                          (n <= st->max_leaf_objects && n < 2u * st->min_leaf_objects);
        if (leaf) {
            M.cls = 0;
        } else if (n <= kSmallMax) {
            M.cls = 1;
            M.list_index = B.n_small++;
        } else if (n <= ctx->medium_max) {
            M.cls = 2;
            M.list_index = B.n_medium++;
        } else {
            M.cls = 3;
            M.list_index = B.n_large++;
            M.tile0 = B.tiles;
            M.ntiles = (n + kTile - 1) / kTile;
            B.tiles += M.ntiles;
        }
    }
    B.toffs[nm] = (uint32_t)total;
    B.noffs[nm] = (uint32_t)slots;
    B.n = (uint32_t)total;
    B.slots = (uint32_t)slots;
    return MGBVH_OK;
}

Params params_of(const mgbvh_ctx* ctx, const mgbvh_settings* st) {
    Params P;
    P.min_leaf = st->min_leaf_objects;
    P.max_leaf = st->max_leaf_objects;
    P.max_depth = st->max_depth;
    P.bins = st->bins;
    P.adaptive_max_n = st->adaptive_max_n;
    P.adaptive_steps = st->adaptive_steps;
    P.medium_max = ctx->medium_max;
    return P;
}

// The persistent build's queue (capacity ctx->qcap, set by run_batch) and
// the median list.
QueueArgs queue_args(mgbvh_ctx* ctx, const Caps& C) {
    QueueArgs Q;
    Q.q = P_<Task>(ctx->q);
    Q.qready = P_<uint32_t>(ctx->qready);
    Q.qcb = P_<uint32_t>(ctx->qcb);
    Q.qcap = ctx->qcap;
    Q.st = P_<QueueState>(ctx->qstate);
    Q.med = P_<Task>(ctx->med_list);
    Q.med_cap = C.tasks;
    Q.wait_ns = ctx->queue_wait_ns;
    return Q;
}

// Device work of a batch on the context's stream. fixed_levels == 0: eager
// (reads level counts back); > 0: capture form, which also copies the slot
// array to the caller's outputs and the counters to pinned host memory.
// queue: the persistent build (one launch over device-side task queues) in
// place of the level passes and subtree launches.
int enqueue_batch(mgbvh_ctx* ctx, const BatchPlan& B, const Caps& C, const mgbvh_settings* st,
                  uint32_t fixed_levels, mgbvh_node* d_nodes, uint32_t* d_lens, uint32_t* d_perm,
                  uint32_t& launches, uint32_t& levels, bool direct, bool queue) {
    const cudaStream_t sm = ctx->stream;
    const uint32_t nm = B.nm, n = B.n;
    const Params P = params_of(ctx, st);
    // pinned staging: counters, mesh records, object offsets, node offsets
    unsigned char* pin = static_cast<unsigned char*>(ctx->pin);
    Counters* h_init = reinterpret_cast<Counters*>(pin);
    DevMesh* h_mesh = reinterpret_cast<DevMesh*>(pin + sizeof(Counters));
    uint32_t* h_toffs = reinterpret_cast<uint32_t*>(h_mesh + nm);
    uint32_t* h_noffs = h_toffs + (nm + 1);
    Counters* d_ctr = P_<Counters>(ctx->ctr);
    MG_CUDA(cudaMemcpyAsync(d_ctr, h_init, sizeof(Counters), cudaMemcpyHostToDevice, sm));
    MG_CUDA(cudaMemcpyAsync(ctx->mesh_buf.p, h_mesh, sizeof(DevMesh) * (size_t)nm,
                            cudaMemcpyHostToDevice, sm));
    MG_CUDA(cudaMemcpyAsync(ctx->toff_buf.p, h_toffs, 4ull * (nm + 1), cudaMemcpyHostToDevice, sm));
    MG_CUDA(cudaMemcpyAsync(ctx->noff_buf.p, h_noffs, 4ull * (nm + 1), cudaMemcpyHostToDevice, sm));
    MG_CUDA(cudaMemsetAsync(ctx->used.p, 0, (size_t)C.nodes, sm));
    Out O;
    // direct: the caller's buffers hold every slot; nodes (and lens) go there
    O.nodes = direct ? d_nodes : P_<mgbvh_node>(ctx->nodes);
    O.lens = (direct && d_lens) ? d_lens : P_<uint32_t>(ctx->lens);
    O.used = P_<uint8_t>(ctx->used);
    O.perm = d_perm;
    O.ctr = d_ctr;
    O.node_cap = C.nodes;
    Rec* rec0 = P_<Rec>(ctx->rec[0]);
    Rec* rec1 = P_<Rec>(ctx->rec[1]);
    const DevMesh* dmesh = P_<DevMesh>(ctx->mesh_buf);
    // timing events are recorded outside a captured graph (around its launch)
    if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->ev0, sm));
    init_mkeys_kernel<<<std::max(1u, std::min((12 * nm + 255) / 256, 1024u)), 256, 0, sm>>>(
        P_<uint32_t>(ctx->mkeys), nm);
    prep_batch_kernel<<<(int)std::min<uint32_t>((n + 255) / 256, 148u * 8u), 256, 0, sm>>>(
        dmesh, P_<uint32_t>(ctx->toff_buf), nm, n, rec0, P_<uint32_t>(ctx->mkeys), d_ctr);
    levels = 0;
    if (queue) {
        // the persistent build: roots into the queues, then one launch
        QueueArgs Q = queue_args(ctx, C);
        MG_CUDA(cudaMemsetAsync(ctx->qstate.p, 0, sizeof(QueueState), sm));
        MG_CUDA(cudaMemsetAsync(ctx->qready.p, 0, 4ull * Q.qcap, sm));
        // queue_hold: tasks counted as pending that never arrive (the test of
        // the bounded waits: the launch must end with a time-out)
        queue_roots_kernel<<<std::max(1u, std::min((nm + 7) / 8, 1024u)), 256, 0, sm>>>(
            dmesh, nm, P_<uint32_t>(ctx->mkeys), Q, O, st->max_depth, P.medium_max, ctx->queue_hold);
        MG_CUDA(cudaGetLastError());
        if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->evp[0], sm));
        const bool small_cap = P.medium_max <= kMediumSmallCap;
        const bool lv = P.adaptive_steps == 0 && P.adaptive_max_n == kSmallMax;
        const size_t smem = small_cap ? sizeof(MediumSmemQ<kMediumSmallCap>) : sizeof(MediumSmemQ<kMediumMax>);
        int grid = small_cap ? ctx->queue_ctas[0] : ctx->queue_ctas[1];
        if (ctx->queue_per_sm) grid = std::min(grid, ctx->sm_count * (int)ctx->queue_per_sm);
        if (small_cap && lv)
            queue_build_kernel<kMediumSmallCap, true><<<grid, kMediumThreads, smem, sm>>>(Q, rec0, rec1, P, O);
        else if (small_cap)
            queue_build_kernel<kMediumSmallCap, false><<<grid, kMediumThreads, smem, sm>>>(Q, rec0, rec1, P, O);
        else if (lv)
            queue_build_kernel<kMediumMax, true><<<grid, kMediumThreads, smem, sm>>>(Q, rec0, rec1, P, O);
        else
            queue_build_kernel<kMediumMax, false><<<grid, kMediumThreads, smem, sm>>>(Q, rec0, rec1, P, O);
        MG_CUDA(cudaGetLastError());
        if (!fixed_levels) {
            MG_CUDA(cudaEventRecord(ctx->evp[1], sm));
            MG_CUDA(cudaEventRecord(ctx->evp[2], sm));
        }
        launches = 4;
        MG_CUDA(cudaMemcpyAsync(ctx->h_qstate, ctx->qstate.p, sizeof(QueueState), cudaMemcpyDeviceToHost, sm));
    } else {
        init_roots_kernel<<<std::max(1u, std::min((nm + 7) / 8, 1024u)), 256, 0, sm>>>(
            dmesh, nm, P_<uint32_t>(ctx->mkeys), P_<Task>(ctx->tasks[0]), P_<uint32_t>(ctx->bins[0]),
            P_<uint32_t>(ctx->cbkeys[0]), P_<uint32_t>(ctx->tile_task[0]), P_<uint32_t>(ctx->tile_begin[0]),
            P_<Task>(ctx->medium), P_<Task>(ctx->small), O, st->max_depth);
        MG_CUDA(cudaGetLastError());
        if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->evp[0], sm));
        launches = 3;
        int rc = run_pipeline(ctx, C, P, O, rec0, rec1, B.n_large > 0, fixed_levels, launches, levels);
        if (rc != MGBVH_OK) return rc;
    }
    if (!fixed_levels) MG_CUDA(cudaEventRecord(ctx->ev1, sm));
    if (fixed_levels && !direct) {
        MG_CUDA(cudaMemcpyAsync(d_nodes, ctx->nodes.p, sizeof(mgbvh_node) * (size_t)B.slots,
                                cudaMemcpyDeviceToDevice, sm));
        if (d_lens)
            MG_CUDA(cudaMemcpyAsync(d_lens, ctx->lens.p, 4ull * B.slots, cudaMemcpyDeviceToDevice, sm));
    }
    MG_CUDA(cudaMemcpyAsync(ctx->h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, sm));
    return MGBVH_OK;
}

bool same_signature(const mgbvh_ctx* ctx, const std::vector<unsigned char>& sig) {
    return ctx->graph_exec && ctx->graph_sig == sig;
}

int run_batch(mgbvh_ctx* ctx, const mgbvh_mesh_desc* meshes, uint32_t nm, const mgbvh_settings* st,
              mgbvh_node* d_nodes, uint32_t cap, uint32_t* d_lens, uint32_t* d_perm,
              uint32_t* out_offsets, mgbvh_stats* stats) {
    const cudaStream_t sm = ctx->stream;
    int rc;
    BatchPlan B;
    if ((rc = plan_batch(ctx, meshes, nm, st, B)) != MGBVH_OK) return rc;
    if (B.n == 0) {
        for (uint32_t m = 0; m <= nm; ++m) out_offsets[m] = 0;
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return MGBVH_WARN_EMPTY;
    }
    const uint32_t n = B.n;
    const Caps C = caps_for(n, ctx->medium_max, nm, B.slots);
#define ENS(buf, bytes) \
    if ((rc = ensure(ctx, buf, (bytes))) != MGBVH_OK) return rc
    ENS(ctx->rec[0], sizeof(Rec) * (size_t)n);
    ENS(ctx->rec[1], sizeof(Rec) * (size_t)n);
    for (int i = 0; i < 2; ++i) {
        ENS(ctx->tasks[i], sizeof(Task) * (size_t)C.tasks);
        ENS(ctx->bins[i], 4ull * kBinWords * C.tasks);
        ENS(ctx->cbkeys[i], 24ull * C.tasks);
        ENS(ctx->tile_task[i], 4ull * C.tiles);
        ENS(ctx->tile_begin[i], 4ull * C.tiles);
    }
    ENS(ctx->tile_hist, 4ull * 96 * C.tiles);
    ENS(ctx->tile_lt, 4ull * C.tiles);
    ENS(ctx->bincode, 2ull * n);
    ENS(ctx->dec, sizeof(Decision) * (size_t)C.tasks);
    ENS(ctx->med_list, sizeof(Task) * (size_t)C.tasks);
    ENS(ctx->medium, sizeof(Task) * (size_t)C.medium);
    ENS(ctx->small, sizeof(Task) * (size_t)C.small);
    ENS(ctx->nodes, sizeof(mgbvh_node) * (size_t)C.nodes);
    ENS(ctx->lens, 4ull * C.nodes);
    ENS(ctx->used, (size_t)C.nodes);
    ENS(ctx->ctr, sizeof(Counters));
    ENS(ctx->mesh_buf, sizeof(DevMesh) * (size_t)nm);
    ENS(ctx->toff_buf, 4ull * (nm + 1));
    ENS(ctx->noff_buf, 4ull * (nm + 1));
    ENS(ctx->mkeys, 48ull * nm);
    if (ctx->learn_w) {
        ENS(ctx->lref, sizeof(LvlRefine) * (size_t)C.tasks);
        ENS(ctx->rbins, 4ull * kRBinWords * C.tasks);
        ENS(ctx->tile_hist2, 4ull * 34 * C.tiles);
    }
    // the persistent build: plain builds (the learned form and sample output
    // run in the level passes) of meshes up to kQueueMaxMesh objects (one CTA
    // splits a node, so a larger root would lengthen the launch's critical path)
    uint32_t max_mesh = 0;
    for (const DevMesh& M : B.hm) max_mesh = std::max(max_mesh, M.n);
    const bool use_queue = ctx->batch_queue && !ctx->learn_w && !ctx->learn_samples && max_mesh <= kQueueMaxMesh;
    // tasks: the roots, and two children per node above medium_max (> 32
    // objects), whose nodes form binary trees with disjoint leaves of > 32
    // objects: at most 2 * (2n / 33) of them
    const uint32_t qcap = 4u * (n / (kSmallMax + 1)) + nm + 8u;
    if (use_queue) {
        ENS(ctx->q, sizeof(Task) * (size_t)qcap);
        ENS(ctx->qready, 4ull * qcap);
        ENS(ctx->qcb, 24ull * qcap);
        ENS(ctx->qstate, sizeof(QueueState));
    }
    ctx->qcap = qcap;
#undef ENS
    if (B.n_large > C.tasks || B.tiles > C.tiles || B.n_medium > C.medium || B.n_small > C.small)
        return fail(ctx, MGBVH_ERR_CAPACITY, "batch root lists exceed their capacity");
    // pinned staging of the plan
    const size_t pin_bytes = sizeof(Counters) + sizeof(DevMesh) * (size_t)nm + 8ull * (nm + 1);
    if (ctx->pin_bytes < pin_bytes) {
        // a graph captured against the old staging must not be replayed
        if (ctx->graph_exec) {
            cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = nullptr;
            ctx->graph_sig.clear();
        }
        if (ctx->pin) cudaFreeHost(ctx->pin);
        ctx->pin = nullptr;
        ctx->pin_bytes = 0;
        MG_CUDA(cudaMallocHost(&ctx->pin, pin_bytes));
        ctx->pin_bytes = pin_bytes;
    }
    {
        unsigned char* pin = static_cast<unsigned char*>(ctx->pin);
        Counters init;
        std::memset(&init, 0, sizeof(init));
        if (!use_queue) {  // the persistent build pushes its roots itself
            init.lvl[0][0] = B.n_large;
            init.lvl[0][1] = B.tiles;
            init.n_medium = B.n_medium;
            init.n_small = B.n_small;
        }
        std::memcpy(pin, &init, sizeof(init));
        std::memcpy(pin + sizeof(Counters), B.hm.data(), sizeof(DevMesh) * (size_t)nm);
        uint32_t* t = reinterpret_cast<uint32_t*>(pin + sizeof(Counters) + sizeof(DevMesh) * (size_t)nm);
        std::memcpy(t, B.toffs.data(), 4ull * (nm + 1));
        std::memcpy(t + nm + 1, B.noffs.data(), 4ull * (nm + 1));
    }
    // signature of everything a captured graph bakes in
    std::vector<unsigned char> sig;
    if (ctx->graph_mode) {
        auto put = [&](const void* p, size_t k) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            sig.insert(sig.end(), c, c + k);
        };
        put(meshes, sizeof(mgbvh_mesh_desc) * (size_t)nm);
        put(st, sizeof(*st));
        put(&ctx->medium_max, 4);
        put(&d_nodes, sizeof(d_nodes));
        put(&d_lens, sizeof(d_lens));
        put(&d_perm, sizeof(d_perm));
        put(&cap, 4);
        put(&ctx->stream, sizeof(ctx->stream));
        put(&use_queue, sizeof(use_queue));
        put(&ctx->queue_hold, 4);
        put(&ctx->queue_wait_ns, sizeof(ctx->queue_wait_ns));
        put(&ctx->small_threads, 4);
        put(&ctx->small_warps, 4);
        put(&ctx->queue_per_sm, 4);
    }
    uint32_t launches = 0, levels = 0;
    bool done = false;
    bool from_graph = false;
    bool had_medians = false;
    if (ctx->graph_mode && same_signature(ctx, sig)) {
        MG_CUDA(cudaEventRecord(ctx->ev0, sm));
        MG_CUDA(cudaGraphLaunch(ctx->graph_exec, sm));
        MG_CUDA(cudaEventRecord(ctx->ev1, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
        const Counters& hc = *ctx->h_ctr;
        // the spare level must have found nothing to do, and no node may wait
        // for a forced median (the graph holds no median passes)
        if (!hc.error && hc.lvl[ctx->graph_levels % 3u][0] == 0 && hc.n_med == 0) {
            done = true;
            from_graph = true;
            launches = ctx->graph_launches;
            levels = ctx->graph_levels;
        }
    }
    auto queue_timed_out = [&]() {
        return use_queue && static_cast<const QueueState*>(ctx->h_qstate)->timeouts != 0;
    };
    if (done && queue_timed_out()) done = false;
    if (!done) {
        if ((rc = enqueue_batch(ctx, B, C, st, 0, d_nodes, d_lens, d_perm, launches, levels,
                                cap >= B.slots, use_queue)) != MGBVH_OK)
            return rc;
        MG_CUDA(cudaStreamSynchronize(sm));
        if (queue_timed_out())
            return fail(ctx, MGBVH_ERR_TIMEOUT,
                        "a wait of the persistent batched build ran out (no task arrived within the wait limit)");
        if (!ctx->h_ctr->error && ctx->h_ctr->n_med) {
            // level-pass nodes that need the forced median
            had_medians = true;
            const bool dir = cap >= B.slots;
            Out O;
            O.nodes = dir ? d_nodes : P_<mgbvh_node>(ctx->nodes);
            O.lens = (dir && d_lens) ? d_lens : P_<uint32_t>(ctx->lens);
            O.used = P_<uint8_t>(ctx->used);
            O.perm = d_perm;
            O.ctr = P_<Counters>(ctx->ctr);
            O.node_cap = C.nodes;
            if ((rc = run_medians(ctx, C, params_of(ctx, st), O, P_<Rec>(ctx->rec[0]), P_<Rec>(ctx->rec[1]), n,
                                  launches)) != MGBVH_OK)
                return rc;
            MG_CUDA(cudaEventRecord(ctx->ev1, sm));
            MG_CUDA(cudaStreamSynchronize(sm));
        }
    }
    const Counters hc = *ctx->h_ctr;
    if (hc.error) return fail(ctx, (int)hc.error, site_text(hc.error_site));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) != cudaSuccess) {
        ms = 0.0f;
        cudaGetLastError();
    }
    const std::vector<uint32_t>& noffs = B.noffs;
    uint32_t count = B.slots;
    const bool direct = cap >= B.slots;
    if (hc.holes > 0) {
        if (direct) {  // the compaction reads the slots from scratch
            MG_CUDA(cudaMemcpyAsync(ctx->nodes.p, d_nodes, sizeof(mgbvh_node) * (size_t)C.nodes,
                                    cudaMemcpyDeviceToDevice, sm));
            if (d_lens)
                MG_CUDA(cudaMemcpyAsync(ctx->lens.p, d_lens, 4ull * C.nodes, cudaMemcpyDeviceToDevice, sm));
        }
        if ((rc = ensure(ctx, ctx->newidx, 4ull * C.nodes)) != MGBVH_OK) return rc;
        if ((rc = ensure(ctx, ctx->widened, 4ull * C.nodes)) != MGBVH_OK) return rc;
        widen_used_kernel<<<std::min<uint32_t>((C.nodes + 255) / 256, 4096u), 256, 0, sm>>>(
            P_<uint8_t>(ctx->used), C.nodes, P_<uint32_t>(ctx->widened));
        size_t tmp = 0;
        MG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, P_<uint32_t>(ctx->widened),
                                              P_<uint32_t>(ctx->newidx), C.nodes, sm));
        if ((rc = ensure(ctx, ctx->cub_tmp, tmp)) != MGBVH_OK) return rc;
        MG_CUDA(cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, tmp, P_<uint32_t>(ctx->widened),
                                              P_<uint32_t>(ctx->newidx), C.nodes, sm));
        std::vector<uint32_t> nidx(C.nodes);
        MG_CUDA(cudaMemcpyAsync(nidx.data(), ctx->newidx.p, 4ull * C.nodes, cudaMemcpyDeviceToHost, sm));
        uint8_t last_used = 0;
        MG_CUDA(cudaMemcpyAsync(&last_used, P_<uint8_t>(ctx->used) + (C.nodes - 1), 1,
                                cudaMemcpyDeviceToHost, sm));
        MG_CUDA(cudaStreamSynchronize(sm));
        count = nidx[C.nodes - 1] + last_used;
        for (uint32_t m = 0; m < nm; ++m) out_offsets[m] = noffs[m] < C.nodes ? nidx[noffs[m]] : count;
        out_offsets[nm] = count;
        if (count > cap) return fail(ctx, MGBVH_ERR_CAPACITY, "node_capacity is smaller than the trees");
        compact_batch_kernel<<<std::min<uint32_t>((C.nodes + 255) / 256, 4096u), 256, 0, sm>>>(
            P_<mgbvh_node>(ctx->nodes), P_<uint32_t>(ctx->lens), P_<uint8_t>(ctx->used),
            P_<uint32_t>(ctx->newidx), P_<uint32_t>(ctx->noff_buf), nm, C.nodes, d_nodes, d_lens);
        MG_CUDA(cudaGetLastError());
    } else {
        if (count > cap) return fail(ctx, MGBVH_ERR_CAPACITY, "node_capacity is smaller than the trees");
        for (uint32_t m = 0; m <= nm; ++m) out_offsets[m] = noffs[m];
        if (!from_graph && !direct) {
            MG_CUDA(cudaMemcpyAsync(d_nodes, ctx->nodes.p, sizeof(mgbvh_node) * (size_t)count,
                                    cudaMemcpyDeviceToDevice, sm));
            if (d_lens)
                MG_CUDA(cudaMemcpyAsync(d_lens, ctx->lens.p, 4ull * count, cudaMemcpyDeviceToDevice, sm));
        }
    }
    MG_CUDA(cudaStreamSynchronize(sm));
    // capture a graph for the next build of this mesh set
    if (ctx->graph_mode && !from_graph && !had_medians && hc.holes == 0 && cap >= B.slots) {
        if (ctx->graph_exec) {
            cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = nullptr;
        }
        ctx->graph_sig.clear();
        cudaGraph_t g = nullptr;
        uint32_t gl = 0, glev = 0;
        const uint32_t fixed = (B.n_large > 0 ? levels : 0) + 1;
        // (capture is not possible on the legacy default stream: then no graph)
        if (cudaStreamBeginCapture(sm, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
        } else {
        const int erc = enqueue_batch(ctx, B, C, st, fixed, d_nodes, d_lens, d_perm, gl, glev, true, use_queue);
        const cudaError_t ce = cudaStreamEndCapture(sm, &g);
        if (erc == MGBVH_OK && ce == cudaSuccess && g) {
            if (cudaGraphInstantiate(&ctx->graph_exec, g, 0) == cudaSuccess) {
                ctx->graph_sig = sig;
                ctx->graph_levels = fixed;
                ctx->graph_launches = gl;
            } else {
                ctx->graph_exec = nullptr;
            }
        }
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        }
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->construction_time = ms * 1e-3;
        stats->node_count = count;
        stats->total_object_count = n;
        stats->height = hc.height;
        stats->max_depth = st->max_depth;
        stats->median_splits = hc.median_splits;
        stats->learned_splits = hc.learned;
        stats->depth_capped_leaves = hc.depth_capped;
        stats->kernel_launches = launches;
        stats->levels = levels;
        const uint32_t MIN = st->min_leaf_objects, MAX = st->max_leaf_objects;
        stats->feasible = MIN == MAX ? 1u : (MAX >= 2 * MIN - 1);
        float pm[4] = {0.f, 0.f, 0.f, 0.f};
        if (!from_graph) {  // phases are not timed inside a graph
            cudaEventElapsedTime(&pm[0], ctx->ev0, ctx->evp[0]);
            cudaEventElapsedTime(&pm[1], ctx->evp[0], ctx->evp[1]);
            cudaEventElapsedTime(&pm[2], ctx->evp[1], ctx->evp[2]);
            cudaEventElapsedTime(&pm[3], ctx->evp[2], ctx->ev1);
            cudaGetLastError();
        }
        for (int i = 0; i < 4; ++i) stats->phase_seconds[i] = pm[i] * 1e-3;
        stats->graph_replay = from_graph ? 1u : 0u;
    }
    return MGBVH_OK;
}

int check_ctx(mgbvh_ctx* ctx) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, MGBVH_ERR_CUDA, cudaGetErrorString(e));
    return MGBVH_OK;
}

int build_common(mgbvh_ctx* ctx, const Input& in_dev, const mgbvh_settings* s, mgbvh_node* d_nodes,
                 uint32_t cap, uint32_t* out_count, uint32_t* d_lens, uint32_t* d_perm,
                 mgbvh_stats* stats) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = validate_settings(ctx, s)) != MGBVH_OK) return rc;
    if (!out_count) return fail(ctx, MGBVH_ERR_INVALID_ARG, "out_node_count is NULL");
    *out_count = 0;
    if (in_dev.n == 0) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return MGBVH_WARN_EMPTY;
    }
    if (!d_nodes || !d_perm) return fail(ctx, MGBVH_ERR_INVALID_ARG, "output pointer is NULL");
    return run_build(ctx, in_dev, s, d_nodes, cap, d_lens, d_perm, out_count, stats);
}

// Host-pointer builds: copy inputs in, build into scratch, copy results out.
// Page-locked host memory (cudaMallocHost, cudaHostAlloc, cudaHostRegister):
// copies from the device into it run asynchronously.
bool host_page_locked(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

int build_host(mgbvh_ctx* ctx, Input in, const mgbvh_settings* s, mgbvh_node* out_nodes, uint32_t cap,
               uint32_t* out_count, uint32_t* out_lens, uint32_t* out_perm, mgbvh_stats* stats) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = validate_settings(ctx, s)) != MGBVH_OK) return rc;
    if (!out_count) return fail(ctx, MGBVH_ERR_INVALID_ARG, "out_node_count is NULL");
    *out_count = 0;
    if (in.n == 0) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return MGBVH_WARN_EMPTY;
    }
    if (!out_nodes || !out_perm) return fail(ctx, MGBVH_ERR_INVALID_ARG, "output pointer is NULL");
    const cudaStream_t sm = ctx->stream;
    Input d = in;
    if (in.kind == kIndexed) {
        if ((rc = ensure(ctx, ctx->in_a, (size_t)in.nverts * in.stride_bytes))) return rc;
        if ((rc = ensure(ctx, ctx->in_b, 12ull * in.n))) return rc;
        MG_CUDA(cudaMemcpyAsync(ctx->in_a.p, in.verts, (size_t)in.nverts * in.stride_bytes,
                                cudaMemcpyHostToDevice, sm));
        MG_CUDA(cudaMemcpyAsync(ctx->in_b.p, in.tris, 12ull * in.n, cudaMemcpyHostToDevice, sm));
        d.verts = P_<float>(ctx->in_a);
        d.tris = P_<uint32_t>(ctx->in_b);
    } else {
        if ((rc = ensure(ctx, ctx->in_a, 24ull * in.n))) return rc;
        MG_CUDA(cudaMemcpyAsync(ctx->in_a.p, in.aabbs, 24ull * in.n, cudaMemcpyHostToDevice, sm));
        d.aabbs = P_<float>(ctx->in_a);
    }
    const uint32_t full = 2 * in.n - 1;
    if ((rc = ensure(ctx, ctx->out_nodes, sizeof(mgbvh_node) * (size_t)full))) return rc;
    if ((rc = ensure(ctx, ctx->out_lens, 4ull * full))) return rc;
    if ((rc = ensure(ctx, ctx->perm, 4ull * in.n))) return rc;
    // page-locked node (and lens) arrays with room for every slot take the
    // nodes in chunks while the subtree kernels still run (run_pipeline)
    const bool stream = cap >= full && host_page_locked(out_nodes) && (!out_lens || host_page_locked(out_lens));
    if (stream && !ctx->cstream) {
        MG_CUDA(cudaStreamCreateWithFlags(&ctx->cstream, cudaStreamNonBlocking));
        for (cudaEvent_t& e : ctx->evs) MG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    ctx->h_nodes_out = stream ? out_nodes : nullptr;
    ctx->h_lens_out = stream ? out_lens : nullptr;
    ctx->streamed = false;
    uint32_t count = 0;
    rc = run_build(ctx, d, s, P_<mgbvh_node>(ctx->out_nodes), full, P_<uint32_t>(ctx->out_lens),
                   P_<uint32_t>(ctx->perm), &count, stats);
    ctx->h_nodes_out = nullptr;
    ctx->h_lens_out = nullptr;
    // no chunk copy may still be writing the caller's arrays after this call
    if (ctx->streamed) MG_CUDA(cudaStreamSynchronize(ctx->cstream));
    if (rc < 0) return rc;
    if (count > cap) return fail(ctx, MGBVH_ERR_CAPACITY, "node_capacity is smaller than the tree");
    // the streamed chunks are the result when no slot was compacted away
    if (!(ctx->streamed && count == full)) {
        MG_CUDA(cudaMemcpyAsync(out_nodes, ctx->out_nodes.p, sizeof(mgbvh_node) * (size_t)count,
                                cudaMemcpyDeviceToHost, sm));
        if (out_lens)
            MG_CUDA(cudaMemcpyAsync(out_lens, ctx->out_lens.p, 4ull * count, cudaMemcpyDeviceToHost, sm));
    }
    MG_CUDA(cudaMemcpyAsync(out_perm, ctx->perm.p, 4ull * in.n, cudaMemcpyDeviceToHost, sm));
    MG_CUDA(cudaStreamSynchronize(sm));
    *out_count = count;
    return rc;
}

Input make_indexed(const float* v, uint32_t stride, uint32_t nv, const uint32_t* t, uint32_t n) {
    Input in;
    in.kind = kIndexed;
    in.verts = v;
    in.stride_bytes = stride;
    in.nverts = nv;
    in.tris = t;
    in.aabbs = nullptr;
    in.n = n;
    return in;
}

Input make_aabbs(const float* a, uint32_t n) {
    Input in;
    in.kind = kAabbs;
    in.verts = nullptr;
    in.stride_bytes = 0;
    in.nverts = 0;
    in.tris = nullptr;
    in.aabbs = a;
    in.n = n;
    return in;
}

int check_indexed_args(mgbvh_ctx* ctx, const float* v, uint32_t stride, const uint32_t* t, uint32_t n) {
    if (n == 0) return MGBVH_OK;
    if (!v || !t) return fail(ctx, MGBVH_ERR_INVALID_ARG, "vertices/triangles pointer is NULL");
    if (stride < 12 || stride % 4) return fail(ctx, MGBVH_ERR_INVALID_ARG, "vertex stride must be >= 12 and a multiple of 4");
    return MGBVH_OK;
}

}  // namespace

extern "C" {

void mgbvh_default_settings(mgbvh_settings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->min_leaf_objects = 1;
    s->max_leaf_objects = 1;
    s->max_depth = 32;
    s->has_bounds = 0;
    s->bins = 0;
    s->adaptive_max_n = 32;
    s->adaptive_steps = 0;
    s->profiling_info = 0;
}

int mgbvh_create(int device, mgbvh_ctx** out_ctx) {
    if (!out_ctx) return MGBVH_ERR_INVALID_ARG;
    *out_ctx = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return MGBVH_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return MGBVH_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MGBVH_ERR_CUDA;
    mgbvh_ctx* ctx = new mgbvh_ctx();
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaEventCreate(&ctx->evp[0]) != cudaSuccess || cudaEventCreate(&ctx->evp[1]) != cudaSuccess ||
        cudaEventCreate(&ctx->evp[2]) != cudaSuccess ||
        cudaMallocHost(&ctx->h_ctr, sizeof(Counters)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_init, sizeof(Counters)) != cudaSuccess ||
        cudaFuncSetAttribute(medium_kernel<false, kMediumMax>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)medium_smem_bytes<false, kMediumMax>()) != cudaSuccess ||
        cudaFuncSetAttribute(medium_kernel<true, kMediumMax>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)medium_smem_bytes<true, kMediumMax>()) != cudaSuccess ||
        cudaFuncSetAttribute(medium_kernel<false, kMediumSmallCap>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)medium_smem_bytes<false, kMediumSmallCap>()) != cudaSuccess ||
        cudaFuncSetAttribute(medium_kernel<true, kMediumSmallCap>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)medium_smem_bytes<true, kMediumSmallCap>()) != cudaSuccess) {
        mgbvh_destroy(ctx);
        return MGBVH_ERR_CUDA;
    }
    std::memset(ctx->h_init, 0, sizeof(Counters));
    for (int i = 0; i < 12; ++i) ctx->h_init->root_keys[i] = ((i % 6) < 3) ? kKeyPosInf : kKeyNegInf;
    ctx->own_stream = true;
    *out_ctx = ctx;
    return MGBVH_OK;
}

void mgbvh_destroy(mgbvh_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    DevBuf* all[] = {&ctx->rec[0], &ctx->rec[1], &ctx->tasks[0], &ctx->tasks[1], &ctx->bins[0],
                     &ctx->bins[1], &ctx->cbkeys[0], &ctx->cbkeys[1], &ctx->tile_task[0],
                     &ctx->tile_task[1], &ctx->tile_begin[0], &ctx->tile_begin[1], &ctx->tile_hist,
                     &ctx->tile_lt, &ctx->dec, &ctx->medium, &ctx->small, &ctx->nodes, &ctx->lens,
                     &ctx->used, &ctx->newidx, &ctx->widened, &ctx->perm, &ctx->ctr, &ctx->cub_tmp, &ctx->in_a,
                     &ctx->in_b, &ctx->out_nodes, &ctx->out_lens, &ctx->mesh_buf,
                     &ctx->toff_buf, &ctx->noff_buf, &ctx->mkeys, &ctx->learn_wt, &ctx->lref,
                     &ctx->rbins, &ctx->tile_hist2, &ctx->med_list, &ctx->med_work, &ctx->med_off,
                     &ctx->med_seg, &ctx->med_keys[0], &ctx->med_keys[1], &ctx->med_vals[0],
                     &ctx->med_vals[1], &ctx->med_flag, &ctx->med_scan, &ctx->q, &ctx->qready,
                     &ctx->qcb, &ctx->qstate, &ctx->bincode};
    for (DevBuf* b : all)
        if (b->p) cudaFree(b->p);
    if (ctx->h_qstate) cudaFreeHost(ctx->h_qstate);
    if (ctx->h_ctr) cudaFreeHost(ctx->h_ctr);
    if (ctx->h_init) cudaFreeHost(ctx->h_init);
    if (ctx->pin) cudaFreeHost(ctx->pin);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    for (cudaEvent_t e : ctx->evs)
        if (e) cudaEventDestroy(e);
    if (ctx->cstream) cudaStreamDestroy(ctx->cstream);
    if (ctx->small2.p) cudaFree(ctx->small2.p);
    if (ctx->medium2.p) cudaFree(ctx->medium2.p);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (cudaEvent_t e : ctx->evp)
        if (e) cudaEventDestroy(e);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int mgbvh_set_stream(mgbvh_ctx* ctx, void* stream) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (stream) {
        ctx->stream = reinterpret_cast<cudaStream_t>(stream);
        ctx->own_stream = false;
    } else {
        cudaSetDevice(ctx->device);
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
            return MGBVH_ERR_CUDA;
        ctx->own_stream = true;
    }
    return MGBVH_OK;
}

const char* mgbvh_last_error(const mgbvh_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

const char* mgbvh_status_string(int status) {
    switch (status) {
        case MGBVH_OK: return "ok";
        case MGBVH_WARN_EMPTY: return "empty object list: empty hierarchy";
        case MGBVH_WARN_INFEASIBLE: return "leaf-size bounds infeasible for this object count";
        case MGBVH_ERR_INVALID_ARG: return "invalid argument";
        case MGBVH_ERR_CAPACITY: return "output capacity too small";
        case MGBVH_ERR_CUDA: return "CUDA error";
        case MGBVH_ERR_TIMEOUT: return "device wait timed out";
        case MGBVH_ERR_ASSERT: return "reference assertion would fail";
        case MGBVH_ERR_UNSUPPORTED: return "unsupported";
        case MGBVH_ERR_NO_DEVICE: return "no CUDA device";
        case MGBVH_ERR_TOO_LARGE:
            return "more objects than the allocation-free build holds (1024)";
        default: return "unknown status";
    }
}

int mgbvh_build_indexed(mgbvh_ctx* ctx, const float* vertices, uint32_t vertex_stride_bytes,
                        uint32_t vertex_count, const uint32_t* triangles, uint32_t triangle_count,
                        const mgbvh_settings* settings, mgbvh_node* out_nodes, uint32_t node_capacity,
                        uint32_t* out_node_count, uint32_t* out_lens, uint32_t* out_perm,
                        mgbvh_stats* out_stats) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    int rc = check_indexed_args(ctx, vertices, vertex_stride_bytes, triangles, triangle_count);
    if (rc) return rc;
    return build_host(ctx, make_indexed(vertices, vertex_stride_bytes, vertex_count, triangles, triangle_count),
                      settings, out_nodes, node_capacity, out_node_count, out_lens, out_perm, out_stats);
}

int mgbvh_build_aabbs(mgbvh_ctx* ctx, const float* aabbs, uint32_t count, const mgbvh_settings* settings,
                      mgbvh_node* out_nodes, uint32_t node_capacity, uint32_t* out_node_count,
                      uint32_t* out_lens, uint32_t* out_perm, mgbvh_stats* out_stats) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (count && !aabbs) return fail(ctx, MGBVH_ERR_INVALID_ARG, "aabbs pointer is NULL");
    return build_host(ctx, make_aabbs(aabbs, count), settings, out_nodes, node_capacity, out_node_count,
                      out_lens, out_perm, out_stats);
}

int mgbvh_build_indexed_dev(mgbvh_ctx* ctx, const float* d_vertices, uint32_t vertex_stride_bytes,
                            uint32_t vertex_count, const uint32_t* d_triangles, uint32_t triangle_count,
                            const mgbvh_settings* settings, mgbvh_node* d_out_nodes,
                            uint32_t node_capacity, uint32_t* out_node_count, uint32_t* d_out_lens,
                            uint32_t* d_out_perm, mgbvh_stats* out_stats) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    int rc = check_indexed_args(ctx, d_vertices, vertex_stride_bytes, d_triangles, triangle_count);
    if (rc) return rc;
    return build_common(ctx, make_indexed(d_vertices, vertex_stride_bytes, vertex_count, d_triangles, triangle_count),
                        settings, d_out_nodes, node_capacity, out_node_count, d_out_lens, d_out_perm,
                        out_stats);
}

int mgbvh_build_aabbs_dev(mgbvh_ctx* ctx, const float* d_aabbs, uint32_t count,
                          const mgbvh_settings* settings, mgbvh_node* d_out_nodes, uint32_t node_capacity,
                          uint32_t* out_node_count, uint32_t* d_out_lens, uint32_t* d_out_perm,
                          mgbvh_stats* out_stats) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (count && !d_aabbs) return fail(ctx, MGBVH_ERR_INVALID_ARG, "aabbs pointer is NULL");
    return build_common(ctx, make_aabbs(d_aabbs, count), settings, d_out_nodes, node_capacity,
                        out_node_count, d_out_lens, d_out_perm, out_stats);
}

int mgbvh_build_batch_dev(mgbvh_ctx* ctx, const mgbvh_mesh_desc* meshes, uint32_t mesh_count,
                          const mgbvh_settings* settings, mgbvh_node* d_out_nodes,
                          uint32_t node_capacity, uint32_t* d_out_lens, uint32_t* d_out_perm,
                          uint32_t* out_node_offsets, mgbvh_stats* out_stats) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = validate_settings(ctx, settings)) != MGBVH_OK) return rc;
    if ((mesh_count && !meshes) || !out_node_offsets)
        return fail(ctx, MGBVH_ERR_INVALID_ARG, "meshes / out_node_offsets is NULL");
    if (!d_out_nodes || !d_out_perm) return fail(ctx, MGBVH_ERR_INVALID_ARG, "output pointer is NULL");
    return run_batch(ctx, meshes, mesh_count, settings, d_out_nodes, node_capacity, d_out_lens,
                     d_out_perm, out_node_offsets, out_stats);
}

int mgbvh_set_split_proposer(mgbvh_ctx* ctx, const void* d_weights_bf16, int gate) {
    if (int rc = check_ctx(ctx)) return rc;
    if (ctx->graph_exec) {  // a captured graph holds the old switch
        cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
        ctx->graph_sig.clear();
    }
    ctx->learn_w = nullptr;
    ctx->learn_gate = gate != 0;
    if (!d_weights_bf16) return MGBVH_OK;
    if (int rc = ensure(ctx, ctx->learn_wt, sizeof(__nv_bfloat16) * mgbvh_mlp::kTParams)) return rc;
    transpose_weights_kernel<<<(mgbvh_mlp::kTParams + 255) / 256, 256, 0, ctx->stream>>>(
        static_cast<const __nv_bfloat16*>(d_weights_bf16), P_<__nv_bfloat16>(ctx->learn_wt));
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaStreamSynchronize(ctx->stream));  // the caller's buffer may go after this
    ctx->learn_w = ctx->learn_wt.p;
    return MGBVH_OK;
}

int mgbvh_set_proposer_gate(mgbvh_ctx* ctx, float refine_threshold, uint32_t min_objects) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (!(refine_threshold == refine_threshold)) return fail(ctx, MGBVH_ERR_INVALID_ARG, "refine_threshold is NaN");
    if (ctx->graph_exec) {  // a captured graph holds the old gate
        cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
        ctx->graph_sig.clear();
    }
    ctx->learn_gate_thr = refine_threshold;
    ctx->learn_min_n = min_objects;
    return MGBVH_OK;
}

int mgbvh_set_sample_output(mgbvh_ctx* ctx, float* d_samples, uint32_t capacity, uint32_t* d_count) {
    if (!ctx || (d_samples && !d_count)) return MGBVH_ERR_INVALID_ARG;
    ctx->learn_samples = d_samples;
    ctx->learn_cap = d_samples ? capacity : 0;
    ctx->learn_count = d_samples ? d_count : nullptr;
    if (ctx->graph_exec) {
        cudaSetDevice(ctx->device);
        cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
        ctx->graph_sig.clear();
    }
    return MGBVH_OK;
}

int mgbvh_set_graph_capture(mgbvh_ctx* ctx, int enable) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    ctx->graph_mode = enable != 0;
    if (!ctx->graph_mode && ctx->graph_exec) {
        cudaSetDevice(ctx->device);
        cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
        ctx->graph_sig.clear();
    }
    return MGBVH_OK;
}

int mgbvh_set_tuning(mgbvh_ctx* ctx, uint32_t medium_max) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (medium_max < kSmallMax + 1 || medium_max > kMediumMax)
        return fail(ctx, MGBVH_ERR_UNSUPPORTED, "medium_max must be 33..1024");
    ctx->medium_max = medium_max;
    return MGBVH_OK;
}

int mgbvh_set_batch_mode(mgbvh_ctx* ctx, int mode) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (mode != MGBVH_BATCH_LEVELS && mode != MGBVH_BATCH_QUEUE)
        return fail(ctx, MGBVH_ERR_INVALID_ARG, "batch mode must be MGBVH_BATCH_LEVELS or MGBVH_BATCH_QUEUE");
    if (mode == MGBVH_BATCH_QUEUE && !ctx->queue_ctas[0]) {
        // shared-memory limits and resident CTAs of the persistent kernel's instances
        const int s_small = (int)sizeof(MediumSmemQ<kMediumSmallCap>), s_big = (int)sizeof(MediumSmemQ<kMediumMax>);
        MG_CUDA(cudaFuncSetAttribute(queue_build_kernel<kMediumSmallCap, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, s_small));
        MG_CUDA(cudaFuncSetAttribute(queue_build_kernel<kMediumSmallCap, false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, s_small));
        MG_CUDA(cudaFuncSetAttribute(queue_build_kernel<kMediumMax, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, s_big));
        MG_CUDA(cudaFuncSetAttribute(queue_build_kernel<kMediumMax, false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, s_big));
        int o[4] = {0, 0, 0, 0};
        MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[0], queue_build_kernel<kMediumSmallCap, true>,
                                                              kMediumThreads, s_small));
        MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[1], queue_build_kernel<kMediumSmallCap, false>,
                                                              kMediumThreads, s_small));
        MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[2], queue_build_kernel<kMediumMax, true>,
                                                              kMediumThreads, s_big));
        MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[3], queue_build_kernel<kMediumMax, false>,
                                                              kMediumThreads, s_big));
        if (!ctx->h_qstate) MG_CUDA(cudaMallocHost(&ctx->h_qstate, sizeof(QueueState)));
        std::memset(ctx->h_qstate, 0, sizeof(QueueState));
        // a grid no larger than what is resident at once: every CTA polls
        ctx->queue_ctas[0] = ctx->sm_count * std::max(1, std::min(o[0], o[1]));
        ctx->queue_ctas[1] = ctx->sm_count * std::max(1, std::min(o[2], o[3]));
    }
    ctx->batch_queue = mode == MGBVH_BATCH_QUEUE;
    return MGBVH_OK;
}

int mgbvh_set_launch_shape(mgbvh_ctx* ctx, uint32_t small_threads, uint32_t queue_ctas_per_sm) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (small_threads == 0) small_threads = 256;
    if (small_threads != 64 && small_threads != 128 && small_threads != 256)
        return fail(ctx, MGBVH_ERR_UNSUPPORTED, "small_threads must be 64, 128 or 256");
    ctx->small_threads = small_threads;
    ctx->queue_per_sm = queue_ctas_per_sm;
    return MGBVH_OK;
}

int mgbvh_set_small_occupancy(mgbvh_ctx* ctx, uint32_t warps_per_sm) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    if (warps_per_sm == 0) warps_per_sm = 24;
    if (warps_per_sm != 16 && warps_per_sm != 24)
        return fail(ctx, MGBVH_ERR_UNSUPPORTED, "small-subtree occupancy must be 16 or 24 warps per SM");
    ctx->small_warps = warps_per_sm;
    return MGBVH_OK;
}

int mgbvh_set_queue_limits(mgbvh_ctx* ctx, uint32_t wait_microseconds, uint32_t held_tasks) {
    if (!ctx) return MGBVH_ERR_INVALID_ARG;
    ctx->queue_wait_ns = wait_microseconds ? 1000ull * wait_microseconds : 2000000000ull;
    ctx->queue_hold = held_tasks;
    return MGBVH_OK;
}

int mgbvh_instance_aabbs_dev(mgbvh_ctx* ctx, const float* d_mesh_bounds, uint32_t mesh_count,
                             const uint32_t* d_instance_mesh, const float* d_transforms,
                             uint32_t instance_count, float* d_out_aabbs) {
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (instance_count == 0) return MGBVH_OK;
    if (!d_mesh_bounds || !d_instance_mesh || !d_transforms || !d_out_aabbs)
        return fail(ctx, MGBVH_ERR_INVALID_ARG, "a device pointer is NULL");
    if ((rc = ensure(ctx, ctx->ctr, sizeof(Counters))) != MGBVH_OK) return rc;
    const cudaStream_t sm = ctx->stream;
    Counters* d_ctr = P_<Counters>(ctx->ctr);
    MG_CUDA(cudaMemsetAsync(d_ctr, 0, 2 * sizeof(uint32_t), sm));  // error, error_site
    const int blocks = (int)std::min<uint32_t>((instance_count + 255) / 256, (uint32_t)ctx->sm_count * 8u);
    instance_aabbs_kernel<<<blocks, 256, 0, sm>>>(d_mesh_bounds, mesh_count, d_instance_mesh, d_transforms,
                                                  instance_count, d_out_aabbs, d_ctr);
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaMemcpyAsync(ctx->h_ctr, d_ctr, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, sm));
    MG_CUDA(cudaStreamSynchronize(sm));
    if (ctx->h_ctr->error) return fail(ctx, (int)ctx->h_ctr->error, site_text(ctx->h_ctr->error_site));
    return MGBVH_OK;
}

int mgbvh_encode_gpu_bytes(const mgbvh_node* nodes, const uint32_t* lens, uint32_t count,
                           uint32_t max_leaf_objects, uint32_t* out_words) {
    if ((count && (!nodes || !out_words)) || max_leaf_objects < 1) return MGBVH_ERR_INVALID_ARG;
    if (max_leaf_objects == 1) {
        std::memcpy(out_words, nodes, sizeof(mgbvh_node) * (size_t)count);
        return MGBVH_OK;
    }
    if (!lens) return MGBVH_ERR_INVALID_ARG;
    // bvh/src/lib.rs:170-195
    uint64_t overflow = 1;
    while (overflow < max_leaf_objects) overflow <<= 1;  // next_power_of_two
    uint32_t len_bits = 0;
    while ((1ull << (len_bits + 1)) <= overflow) ++len_bits;  // ilog2
    if (len_bits >= 32) return MGBVH_ERR_ASSERT;
    const uint32_t child_bits = 32 - len_bits;
    const uint32_t len_mask = (1u << len_bits) - 1u;
    const uint32_t child_mask = ~len_mask;
    for (uint32_t i = 0; i < count; ++i) {
        const mgbvh_node& nd = nodes[i];
        if (nd.child_node == 0 && lens[i] >= overflow) return MGBVH_ERR_ASSERT;
        uint32_t* w = out_words + 8ull * i;
        std::memcpy(w, &nd, 28);
        const uint32_t packed = (child_bits >= 32 ? 0u : ((lens[i] & len_mask) << child_bits)) |
                                (nd.child_node & child_mask);
        w[7] = packed;
    }
    return MGBVH_OK;
}

double mgbvh_sah_cost(const mgbvh_node* nodes, const uint32_t* lens, uint32_t count) {
    if (!nodes || !lens || count == 0) return 0.0;
    auto sa = [](const mgbvh_node& n) {
        const double w = (double)n.max[0] - n.min[0], h = (double)n.max[1] - n.min[1],
                     d = (double)n.max[2] - n.min[2];
        if (w < 0 || h < 0 || d < 0) return 0.0;
        return 2.0 * (w * h + w * d + h * d);
    };
    const double root = sa(nodes[0]);
    if (!(root > 0.0)) return 0.0;
    double c = 0.0;
    for (uint32_t i = 0; i < count; ++i) {
        const double r = sa(nodes[i]) / root;
        c += nodes[i].child_node ? (double)kDepthCost * r : (double)kObjectCost * lens[i] * r;
    }
    return c;
}


// Allocation-free build (see include/mgbvh.h). Every call looks up, for the
// current device and context, the scratch array's device address
// (cudaGetSymbolAddress allocates nothing), the medium kernel's shared-memory
// limit and the SM count: nothing is cached, so a call after a device reset
// never launches on an address of a context that is gone.
int mgbvh_build_aabbs_noalloc(const float* d_aabbs, uint32_t count, const mgbvh_settings* settings,
                              mgbvh_node* d_out_nodes, uint32_t node_capacity,
                              uint32_t* out_node_count, uint32_t* d_out_lens, uint32_t* d_out_perm,
                              void* cuda_stream) {
    if (!out_node_count) return MGBVH_ERR_INVALID_ARG;
    *out_node_count = 0;
    int rc = validate_settings(nullptr, settings);
    if (rc != MGBVH_OK) return rc;
    if (count == 0) return MGBVH_WARN_EMPTY;
    if (count > kNoAllocMax) return MGBVH_ERR_TOO_LARGE;
    if (!d_aabbs || !d_out_nodes || !d_out_perm) return MGBVH_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return MGBVH_ERR_NO_DEVICE;
    void* addr = nullptr;
    int sms = 0;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return MGBVH_ERR_CUDA;
    if (cudaFuncSetAttribute(medium_kernel<false, kMediumMax>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)medium_smem_bytes<false, kMediumMax>()) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return MGBVH_ERR_CUDA;
    NoAllocScratch* S = reinterpret_cast<NoAllocScratch*>(addr);
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(cuda_stream);
    const mgbvh_settings* st = settings;
    const uint32_t n = count, slots = 2 * n - 1;
    Params P;
    P.min_leaf = st->min_leaf_objects;
    P.max_leaf = st->max_leaf_objects;
    P.max_depth = st->max_depth;
    P.bins = st->bins;
    P.adaptive_max_n = st->adaptive_max_n;
    P.adaptive_steps = st->adaptive_steps;
    P.medium_max = kMediumMax;
    Out O;
    O.nodes = S->nodes;
    O.lens = S->lens;
    O.used = S->used;
    O.perm = d_out_perm;
    O.ctr = &S->ctr;
    O.node_cap = slots;
    noalloc_init_kernel<<<1, 256, 0, sm>>>(S, slots);
    prep_aabbs_kernel<<<(n + 255) / 256, 256, 0, sm>>>(d_aabbs, n, S->rec, &S->ctr);
    const bool root_leaf = n <= 1 || st->max_depth == 0 ||
                           (n <= st->max_leaf_objects && n < 2u * st->min_leaf_objects);
    const uint32_t cls = root_leaf ? 0u : (n <= kSmallMax ? 1u : 2u);
    const float* bb = st->bounds;
    init_root_kernel<<<(n + 255) / 256, 256, 0, sm>>>(n, cls, st->has_bounds, bb[0], bb[1], bb[2],
                                                      bb[3], bb[4], bb[5], nullptr, nullptr, nullptr,
                                                      nullptr, nullptr, S->medium, S->small, O, 0u,
                                                      st->max_depth);
    if (cls == 2)
        medium_kernel<false, kMediumMax><<<1, kMediumThreads, medium_smem_bytes<false, kMediumMax>(), sm>>>(
            S->medium, S->rec, S->rec, S->small, kNoAllocMax / 2 + 8, P, O, Learn{nullptr, 0, nullptr, 0, nullptr},
            nullptr);
    if (cls != 0) {
        const int grid = std::max(1, std::min(sms, (int)((n / 2 + 8 + 7) / 8)));
        if (P.adaptive_steps == 0 && P.adaptive_max_n == kSmallMax)
            small_kernel<true, 3><<<grid, 256, 0, sm>>>(S->small, S->rec, S->rec, P, O, nullptr);
        else
            small_kernel<false, 3><<<grid, 256, 0, sm>>>(S->small, S->rec, S->rec, P, O, nullptr);
    }
    noalloc_finish_kernel<<<1, 1024, 0, sm>>>(S, slots, d_out_nodes, d_out_lens, node_capacity);
    if (cudaGetLastError() != cudaSuccess) return MGBVH_ERR_CUDA;
    struct {
        Counters c;
        uint32_t count;
    } h;
    static_assert(offsetof(NoAllocScratch, count) == offsetof(NoAllocScratch, ctr) + sizeof(Counters),
                  "count follows the counters");
    if (cudaMemcpyAsync(&h, &S->ctr, sizeof(Counters) + 4, cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (h.c.error) return (int)h.c.error;
    *out_node_count = h.count;
    const uint32_t MIN = st->min_leaf_objects, MAX = st->max_leaf_objects;
    const bool feasible = (MIN == MAX) ? (n % MIN == 0) : (MAX >= 2 * MIN - 1);
    return feasible ? MGBVH_OK : MGBVH_WARN_INFEASIBLE;
}

}  // extern "C"
