// mgbvh_trace.cu — closest-hit traversal of a built BVH, and a brute-force
// intersector to check it.
//
// Restates the closest-hit math of marigold's BLAS traversal
// (marigold/assets/shaders/slang/lib/scene.slang:143-220, 296-310) as CUDA:
//   * Moller-Trumbore ray/triangle test with the shader's thresholds:
//     |det| < 1e-6 and t < 1e-6 reject (scene.slang:19-89);
//   * stack traversal, both children tested, the nearer one popped first
//     (far child pushed first, scene.slang:129-134 / 199-204);
//   * leaves: child_node == 0, start_index = first object, one object per
//     leaf unless per-node lengths are given.
// Deliberate differences, so that the traversal can be checked hit for hit
// against brute force: the slab test is conservative (t_far grown by
// 2*gamma(3), PBRT's robust bound) and keeps boxes whose entry equals the
// current closest t; equal hit distances resolve to the lowest triangle index
// (the shader keeps the later-tested one, scene.slang:57-82 via
// intersect.slang's Hit::merge). Hit distances are in ray units; the shader's
// instance-scale quirk (scene.slang:168-169) does not arise in one level.
//
// The library is compiled with -fmad=false: every dot and cross product is
// evaluated as written below, the same way as the CPU cross-check.
//
// Rays are traced in a sorted order (ray_key_kernel + a radix sort, inside
// the timed call): rays that start in nearby cells of the root box and head
// in similar directions share warps, so their lanes walk similar paths
// through the tree and reuse the same nodes in cache. Each ray's result is
// written at its own index; the order changes no hit.

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mgbvh.h"

namespace mgbvh_trace {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr int kStack = 64;  // scene.slang:5-7 (BVH_STACK_SIZE = 32 + 32)
constexpr uint32_t kNoHit = 0xFFFFFFFFu;

struct TriRec {  // one triangle in leaf order: v1 + original index, v2, v3
    float4 a;    // v1.xyz, triangle index (bits)
    float4 b;    // v2.xyz
    float4 c;    // v3.xyz
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// Moller-Trumbore as scene.slang:19-89 evaluates it; returns t or -1 (miss).
__device__ __forceinline__ float intersect_tri(float ox, float oy, float oz, float dx, float dy,
                                               float dz, const TriRec& t) {
    const float e1x = __fsub_rn(t.b.x, t.a.x), e1y = __fsub_rn(t.b.y, t.a.y),
                e1z = __fsub_rn(t.b.z, t.a.z);
    const float e2x = __fsub_rn(t.c.x, t.a.x), e2y = __fsub_rn(t.c.y, t.a.y),
                e2z = __fsub_rn(t.c.z, t.a.z);
    // h = cross(dir, edge2)
    const float hx = __fsub_rn(__fmul_rn(dy, e2z), __fmul_rn(dz, e2y));
    const float hy = __fsub_rn(__fmul_rn(dz, e2x), __fmul_rn(dx, e2z));
    const float hz = __fsub_rn(__fmul_rn(dx, e2y), __fmul_rn(dy, e2x));
    const float det = dot3(hx, hy, hz, e1x, e1y, e1z);
    if (fabsf(det) < 1e-6f) return -1.0f;
    const float f = __fdiv_rn(1.0f, det);
    const float sx = __fsub_rn(ox, t.a.x), sy = __fsub_rn(oy, t.a.y), sz = __fsub_rn(oz, t.a.z);
    const float u = __fmul_rn(f, dot3(sx, sy, sz, hx, hy, hz));
    if (u < 0.0f || u > 1.0f) return -1.0f;
    // q = cross(s, edge1)
    const float qx = __fsub_rn(__fmul_rn(sy, e1z), __fmul_rn(sz, e1y));
    const float qy = __fsub_rn(__fmul_rn(sz, e1x), __fmul_rn(sx, e1z));
    const float qz = __fsub_rn(__fmul_rn(sx, e1y), __fmul_rn(sy, e1x));
    const float v = __fmul_rn(f, dot3(dx, dy, dz, qx, qy, qz));
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return -1.0f;
    const float tt = __fmul_rn(f, dot3(e2x, e2y, e2z, qx, qy, qz));
    if (tt < 1e-6f) return -1.0f;
    return tt;
}

// Conservative slab test: the entry distance if the box can hold a hit at a
// distance <= best, else NaN (which fails every comparison, also with an
// infinite best).
__device__ __forceinline__ float box_entry(float ox, float oy, float oz, float ix, float iy, float iz,
                                           const float4& lo, const float4& hi, float best) {
    const float tx0 = (lo.x - ox) * ix, tx1 = (hi.x - ox) * ix;
    const float ty0 = (lo.y - oy) * iy, ty1 = (hi.y - oy) * iy;
    const float tz0 = (lo.z - oz) * iz, tz1 = (hi.z - oz) * iz;
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    tf *= 1.0000003576278687f;  // 1 + 2 * gamma(3), gamma(n) = n*eps/(1 - n*eps)
    return (tn <= tf && tn <= best) ? tn : __int_as_float(0x7FFFFFFF);
}

struct Counts {
    unsigned long long nodes, boxes, tris;
};

template <bool kLens>
__global__ void __launch_bounds__(128) trace_kernel(const float4* __restrict__ nodes,
                                                    const uint32_t* __restrict__ lens,
                                                    const TriRec* __restrict__ tris,
                                                    const float4* __restrict__ rays, uint32_t n_rays,
                                                    float* __restrict__ hit_t,
                                                    uint32_t* __restrict__ hit_prim, Counts* counts,
                                                    int* err, const uint32_t* __restrict__ order) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t c_nodes = 0, c_boxes = 0, c_tris = 0;
    if (j < n_rays) {
        const uint32_t i = order ? order[j] : j;  // the ray this thread traces
        const float4 o = rays[2 * i], d = rays[2 * i + 1];
        const float ix = __fdiv_rn(1.0f, d.x), iy = __fdiv_rn(1.0f, d.y), iz = __fdiv_rn(1.0f, d.z);
        float best = __int_as_float(0x7F800000);
        uint32_t best_prim = kNoHit;
        uint32_t stack[kStack];
        int sp = 0;
        const float4 rlo = nodes[0], rhi = nodes[1];
        c_boxes++;
        if (box_entry(o.x, o.y, o.z, ix, iy, iz, rlo, rhi, best) <= best) stack[sp++] = 0;
        while (sp > 0) {
            const uint32_t ni = stack[--sp];
            c_nodes++;
            const float4 nhi = nodes[2 * ni + 1];
            const uint32_t child = __float_as_uint(nhi.w);
            if (child != 0) {
                const float4 alo = nodes[2 * child], ahi = nodes[2 * child + 1];
                const float4 blo = nodes[2 * child + 2], bhi = nodes[2 * child + 3];
                c_boxes += 2;
                const float da = box_entry(o.x, o.y, o.z, ix, iy, iz, alo, ahi, best);
                const float db = box_entry(o.x, o.y, o.z, ix, iy, iz, blo, bhi, best);
                const bool pa = da <= best, pb = db <= best;
                if (sp + 2 > kStack) {  // cannot happen for depth <= 62; never overflow
                    atomicExch(err, 1);
                    break;
                }
                if (pa && pb) {
                    const bool a_first = da < db;
                    stack[sp++] = a_first ? child + 1 : child;
                    stack[sp++] = a_first ? child : child + 1;
                } else if (pa || pb) {
                    stack[sp++] = pa ? child : child + 1;
                }
            } else {
                const float4 nlo = nodes[2 * ni];
                const uint32_t start = __float_as_uint(nlo.w);
                const uint32_t len = kLens ? lens[ni] : 1u;
                for (uint32_t k = start; k < start + len; ++k) {
                    const TriRec t = tris[k];
                    c_tris++;
                    const float tt = intersect_tri(o.x, o.y, o.z, d.x, d.y, d.z, t);
                    const uint32_t prim = __float_as_uint(t.a.w);
                    if (tt >= 0.0f && (tt < best || (tt == best && prim < best_prim))) {
                        best = tt;
                        best_prim = prim;
                    }
                }
            }
        }
        hit_t[i] = best_prim == kNoHit ? -1.0f : best;
        hit_prim[i] = best_prim;
    }
    if (counts) {
        // warp totals, one atomic per warp
        unsigned long long a = c_nodes, b = c_boxes, c = c_tris;
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_down_sync(kFull, a, off);
            b += __shfl_down_sync(kFull, b, off);
            c += __shfl_down_sync(kFull, c, off);
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicAdd(&counts->nodes, a);
            atomicAdd(&counts->boxes, b);
            atomicAdd(&counts->tris, c);
        }
    }
}

#ifndef MGBVH_TRACE_PERSISTENT
#define MGBVH_TRACE_PERSISTENT 1  // traversals by persistent warps that refill idle lanes (tuning knob)
#endif
#ifndef MGBVH_TRACE_REFILL
#define MGBVH_TRACE_REFILL 16  // a warp fetches new rays once this many of its lanes are idle (tuning knob;
                                // mixed scene: 68.6 / 71.8 / 69.4 / 65.2 Mrays/s at 8 / 16 / 24 / 28)
#endif

// trace_kernel with persistent warps: every lane holds one ray's traversal
// state and takes one step per round (one node: its children's boxes, or its
// leaf's triangles). Lanes whose ray is done write its hit and go idle; once
// MGBVH_TRACE_REFILL lanes of a warp are idle (or all of them), the warp
// takes that many ray indices from the global counter *next and starts
// them. A warp so keeps most lanes busy instead of running until its longest
// ray ends. Same tests, order of node visits per ray and results as
// trace_kernel.
template <bool kLens>
__global__ void __launch_bounds__(128) trace_persistent_kernel(const float4* __restrict__ nodes,
                                                               const uint32_t* __restrict__ lens,
                                                               const TriRec* __restrict__ tris,
                                                               const float4* __restrict__ rays, uint32_t n_rays,
                                                               float* __restrict__ hit_t,
                                                               uint32_t* __restrict__ hit_prim, Counts* counts,
                                                               int* err, const uint32_t* __restrict__ order,
                                                               uint32_t* __restrict__ next) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t c_nodes = 0, c_boxes = 0, c_tris = 0;
    bool has = false, exhausted = false;
    uint32_t ri = 0, best_prim = kNoHit;
    float ox = 0.f, oy = 0.f, oz = 0.f, dx = 0.f, dy = 0.f, dz = 0.f, ix = 0.f, iy = 0.f, iz = 0.f;
    float best = 0.f;
    uint32_t stack[kStack];
    int sp = 0;
    for (;;) {
        const uint32_t idle = __ballot_sync(kFull, !has);
        if (!exhausted && idle != 0u &&
            (static_cast<uint32_t>(__popc(idle)) >= MGBVH_TRACE_REFILL || idle == kFull)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(next, static_cast<uint32_t>(__popc(idle)));
            base = __shfl_sync(kFull, base, 0);
            if (base >= n_rays) exhausted = true;  // warp-uniform
            if (!has) {
                const uint32_t j = base + static_cast<uint32_t>(__popc(idle & ((1u << lane) - 1u)));
                if (j < n_rays) {
                    ri = order ? order[j] : j;
                    const float4 o = rays[2 * ri], d = rays[2 * ri + 1];
                    ox = o.x, oy = o.y, oz = o.z, dx = d.x, dy = d.y, dz = d.z;
                    ix = __fdiv_rn(1.0f, d.x), iy = __fdiv_rn(1.0f, d.y), iz = __fdiv_rn(1.0f, d.z);
                    best = __int_as_float(0x7F800000);
                    best_prim = kNoHit;
                    sp = 0;
                    const float4 rlo = nodes[0], rhi = nodes[1];
                    c_boxes++;
                    if (box_entry(ox, oy, oz, ix, iy, iz, rlo, rhi, best) <= best) stack[sp++] = 0;
                    has = true;
                }
            }
        }
        if (!__any_sync(kFull, has)) {
            if (exhausted) break;
            continue;  // all lanes idle: the loop's next pass refills them
        }
        if (has && sp > 0) {
            const uint32_t ni = stack[--sp];
            c_nodes++;
            const float4 nhi = nodes[2 * ni + 1];
            const uint32_t child = __float_as_uint(nhi.w);
            if (child != 0) {
                const float4 alo = nodes[2 * child], ahi = nodes[2 * child + 1];
                const float4 blo = nodes[2 * child + 2], bhi = nodes[2 * child + 3];
                c_boxes += 2;
                const float da = box_entry(ox, oy, oz, ix, iy, iz, alo, ahi, best);
                const float db = box_entry(ox, oy, oz, ix, iy, iz, blo, bhi, best);
                const bool pa = da <= best, pb = db <= best;
                if (sp + 2 > kStack) {  // cannot happen for depth <= 62; never overflow
                    atomicExch(err, 1);
                    sp = 0;
                } else if (pa && pb) {
                    const bool a_first = da < db;
                    stack[sp++] = a_first ? child + 1 : child;
                    stack[sp++] = a_first ? child : child + 1;
                } else if (pa || pb) {
                    stack[sp++] = pa ? child : child + 1;
                }
            } else {
                const float4 nlo = nodes[2 * ni];
                const uint32_t start = __float_as_uint(nlo.w);
                const uint32_t len = kLens ? lens[ni] : 1u;
                for (uint32_t k = start; k < start + len; ++k) {
                    const TriRec t = tris[k];
                    c_tris++;
                    const float tt = intersect_tri(ox, oy, oz, dx, dy, dz, t);
                    const uint32_t prim = __float_as_uint(t.a.w);
                    if (tt >= 0.0f && (tt < best || (tt == best && prim < best_prim))) {
                        best = tt;
                        best_prim = prim;
                    }
                }
            }
        }
        if (has && sp == 0) {
            hit_t[ri] = best_prim == kNoHit ? -1.0f : best;
            hit_prim[ri] = best_prim;
            has = false;
        }
    }
    if (counts) {
        unsigned long long a = c_nodes, b = c_boxes, c = c_tris;
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_down_sync(kFull, a, off);
            b += __shfl_down_sync(kFull, b, off);
            c += __shfl_down_sync(kFull, c, off);
        }
        if (lane == 0) {
            atomicAdd(&counts->nodes, a);
            atomicAdd(&counts->boxes, b);
            atomicAdd(&counts->tris, c);
        }
    }
}


// Every ray against every triangle (shared-memory tiles of triangles).
__global__ void __launch_bounds__(256) brute_kernel(const TriRec* __restrict__ tris, uint32_t n_tris,
                                                    const float4* __restrict__ rays, uint32_t n_rays,
                                                    float* __restrict__ hit_t,
                                                    uint32_t* __restrict__ hit_prim) {
    __shared__ TriRec tile[256];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float4 o = make_float4(0.f, 0.f, 0.f, 0.f), d = make_float4(0.f, 0.f, 1.f, 0.f);
    if (i < n_rays) {
        o = rays[2 * i];
        d = rays[2 * i + 1];
    }
    float best = __int_as_float(0x7F800000);
    uint32_t best_prim = kNoHit;
    for (uint32_t base = 0; base < n_tris; base += 256) {
        __syncthreads();
        if (base + threadIdx.x < n_tris) tile[threadIdx.x] = tris[base + threadIdx.x];
        __syncthreads();
        const uint32_t m = min(256u, n_tris - base);
        for (uint32_t k = 0; k < m; ++k) {
            const TriRec& t = tile[k];
            const float tt = intersect_tri(o.x, o.y, o.z, d.x, d.y, d.z, t);
            const uint32_t prim = __float_as_uint(t.a.w);
            if (tt >= 0.0f && (tt < best || (tt == best && prim < best_prim))) {
                best = tt;
                best_prim = prim;
            }
        }
    }
    if (i < n_rays) {
        hit_t[i] = best_prim == kNoHit ? -1.0f : best;
        hit_prim[i] = best_prim;
    }
}

// Triangles in leaf order (the crate's permuted list) with their vertices.
__global__ void gather_kernel(const float* __restrict__ verts, uint32_t stride_floats,
                              uint32_t nverts, const uint32_t* __restrict__ tris,
                              const uint32_t* __restrict__ perm, uint32_t n, TriRec* __restrict__ out,
                              int* err) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t p = perm[k];
        if (p >= n) {
            atomicExch(err, 2);
            continue;
        }
        uint32_t v[3] = {tris[3 * (size_t)p], tris[3 * (size_t)p + 1], tris[3 * (size_t)p + 2]};
        if (v[0] >= nverts || v[1] >= nverts || v[2] >= nverts) {
            atomicExch(err, 2);
            continue;
        }
        const float* a = verts + (size_t)v[0] * stride_floats;
        const float* b = verts + (size_t)v[1] * stride_floats;
        const float* c = verts + (size_t)v[2] * stride_floats;
        TriRec r;
        r.a = make_float4(a[0], a[1], a[2], __uint_as_float(p));
        r.b = make_float4(b[0], b[1], b[2], 0.0f);
        r.c = make_float4(c[0], c[1], c[2], 0.0f);
        out[k] = r;
    }
}


// ---------------------------------------------------------------- wide BVH
//
// An 8-wide BVH with quantized child boxes, collapsed from the binary tree
// (the compressed wide BVH of Ylitie, Karras and Laine, "Efficient Incoherent
// Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017, in a layout
// of this library's own). Each wide node holds up to 8 children, found by
// opening, from the node's two binary children, the internal child of largest
// surface area until 8 children or only leaves remain. Child boxes are stored
// as 8-bit steps on a per-node grid: origin p (the node box's minimum) and a
// power-of-two step per axis, each child box widened outward to whole steps,
// checked in float with the traversal's own dequantization (p + q * step), so
// the stored box always contains the exact one.

constexpr uint32_t kWideLeaf = 0x80000000u;  // ref of a leaf child: first triangle | kWideLeaf
constexpr int kWideStack = 128;

struct WNode {           // 112 bytes
    float px, py, pz;    // grid origin
    uint8_t e[3];        // grid step per axis: 2^(e - 127)
    uint8_t nchild;
    uint8_t qlo[3][8];   // child boxes in grid steps
    uint8_t qhi[3][8];
    uint32_t ref[8];     // wide node index, or first triangle | kWideLeaf
    uint8_t cnt[8];      // triangles of a leaf child
    uint32_t pad[2];
};
static_assert(sizeof(WNode) == 112, "wide node layout");

__device__ __forceinline__ float box_sa(const float4& lo, const float4& hi) {
    const float w = hi.x - lo.x, h = hi.y - lo.y, d = hi.z - lo.z;
    return w * h + w * d + h * d;
}

__device__ __forceinline__ float wstep(uint8_t e) { return __int_as_float(static_cast<uint32_t>(e) << 23); }

__device__ __forceinline__ float wdeq(float p, uint32_t q, float step) {
    return __fadd_rn(p, __fmul_rn(__uint2float_rn(q), step));
}

// One level of the collapse: wide nodes [range[0], range[1]) whose binary
// node is binid[w] with binlen[w] objects; their children that stay internal
// become wide nodes of the next level (slots taken from *counter, their
// binary nodes and lengths recorded in binid/binlen). A child's length comes
// from the start indices (the lt child starts where its parent starts, the
// gt child after the lt child's objects), so the collapse needs no per-node
// lengths. A child of at most kWideLeafMax objects becomes a leaf child over
// its contiguous range of triangles.
#ifndef MGBVH_WIDE_LEAF_MAX
#define MGBVH_WIDE_LEAF_MAX 2  // largest subtree kept as one leaf child (tuning knob)
#endif
constexpr uint32_t kWideLeafMax = MGBVH_WIDE_LEAF_MAX;

__global__ void __launch_bounds__(128) wide_level_kernel(const float4* __restrict__ nodes,
                                                         uint32_t* __restrict__ binid,
                                                         uint32_t* __restrict__ binlen,
                                                         const uint32_t* __restrict__ range,
                                                         uint32_t* __restrict__ counter, WNode* __restrict__ wn,
                                                         uint32_t cap, int* err) {
    const uint32_t begin = range[0], end = range[1];
    for (uint32_t w = begin + blockIdx.x * blockDim.x + threadIdx.x; w < end; w += gridDim.x * blockDim.x) {
        const uint32_t b = binid[w], blen = binlen[w];
        uint32_t c[8], cl[8];
        uint32_t m = 0;
        auto internal = [&](uint32_t node, uint32_t len) {
            return __float_as_uint(nodes[2 * node + 1].w) != 0 && len > kWideLeafMax;
        };
        auto open = [&](uint32_t node, uint32_t len, uint32_t& gt, uint32_t& gl, uint32_t& lt, uint32_t& ll) {
            const uint32_t ch = __float_as_uint(nodes[2 * node + 1].w);
            gt = ch;
            lt = ch + 1;
            ll = __float_as_uint(nodes[2 * ch].w) - __float_as_uint(nodes[2 * (ch + 1)].w);
            gl = len - ll;
        };
        if (!internal(b, blen)) {
            c[0] = b;
            cl[0] = blen;
            m = 1;  // a small root: one leaf child
        } else {
            open(b, blen, c[0], cl[0], c[1], cl[1]);
            m = 2;
            while (m < 8) {
                int pick = -1;
                float psa = -1.0f;
                for (uint32_t j = 0; j < m; ++j) {
                    if (!internal(c[j], cl[j])) continue;
                    const float sa = box_sa(nodes[2 * c[j]], nodes[2 * c[j] + 1]);
                    if (sa > psa) {
                        psa = sa;
                        pick = (int)j;
                    }
                }
                if (pick < 0) break;
                open(c[pick], cl[pick], c[pick], cl[pick], c[m], cl[m]);
                ++m;
            }
        }
        uint32_t nint = 0;
        float4 blo[8], bhi[8];
        float lo[3] = {__int_as_float(0x7F800000), __int_as_float(0x7F800000), __int_as_float(0x7F800000)};
        float hi[3] = {__int_as_float(0xFF800000), __int_as_float(0xFF800000), __int_as_float(0xFF800000)};
        for (uint32_t j = 0; j < m; ++j) {
            blo[j] = nodes[2 * c[j]];
            bhi[j] = nodes[2 * c[j] + 1];
            if (internal(c[j], cl[j])) ++nint;
            lo[0] = fminf(lo[0], blo[j].x);
            lo[1] = fminf(lo[1], blo[j].y);
            lo[2] = fminf(lo[2], blo[j].z);
            hi[0] = fmaxf(hi[0], bhi[j].x);
            hi[1] = fmaxf(hi[1], bhi[j].y);
            hi[2] = fmaxf(hi[2], bhi[j].z);
        }
        const uint32_t base = nint ? atomicAdd(counter, nint) : 0u;
        if (base + nint > cap) {
            atomicExch(err, 3);
            continue;
        }
        WNode out;
        out.px = lo[0];
        out.py = lo[1];
        out.pz = lo[2];
        out.nchild = (uint8_t)m;
        out.pad[0] = out.pad[1] = 0;
        // smallest step 2^k with p + 255 * 2^k >= the node's maximum, per axis
        for (int a = 0; a < 3; ++a) {
            const float ext = __fsub_rn(hi[a], lo[a]);
            int k = -126;
            if (ext > 0.0f) {
                int ex;
                frexpf(__fdiv_rn(ext, 255.0f), &ex);  // ext / 255 < 2^ex
                k = max(ex - 1, -126);
                while (k < 127 && wdeq(lo[a], 255u, wstep((uint8_t)(k + 127))) < hi[a]) ++k;
            }
            out.e[a] = (uint8_t)(k + 127);
        }
        const float p[3] = {lo[0], lo[1], lo[2]};
        uint32_t next = base;
        for (uint32_t j = 0; j < 8; ++j) {
            if (j >= m) {
                for (int a = 0; a < 3; ++a) out.qlo[a][j] = out.qhi[a][j] = 0;
                out.ref[j] = 0;
                out.cnt[j] = 0;
                continue;
            }
            const float cl3[3] = {blo[j].x, blo[j].y, blo[j].z}, ch3[3] = {bhi[j].x, bhi[j].y, bhi[j].z};
            for (int a = 0; a < 3; ++a) {
                const float st = wstep(out.e[a]);
                const float ql = floorf(__fdiv_rn(__fsub_rn(cl3[a], p[a]), st));
                const float qh = ceilf(__fdiv_rn(__fsub_rn(ch3[a], p[a]), st));
                uint32_t qa = (uint32_t)fminf(fmaxf(ql, 0.0f), 255.0f);
                uint32_t qb = (uint32_t)fminf(fmaxf(qh, 0.0f), 255.0f);
                while (qa > 0 && wdeq(p[a], qa, st) > cl3[a]) --qa;
                while (qb < 255 && wdeq(p[a], qb, st) < ch3[a]) ++qb;
                out.qlo[a][j] = (uint8_t)qa;
                out.qhi[a][j] = (uint8_t)qb;
            }
            if (internal(c[j], cl[j])) {
                out.ref[j] = next;
                out.cnt[j] = 0;
                binid[next] = c[j];
                binlen[next] = cl[j];
                ++next;
            } else {
                if (cl[j] > 255u) atomicExch(err, 4);
                out.ref[j] = __float_as_uint(blo[j].w) | kWideLeaf;
                out.cnt[j] = (uint8_t)min(cl[j], 255u);
            }
        }
        wn[w] = out;
    }
}

// The next level's range: the slots taken by the level that just ran.
__global__ void wide_advance_kernel(const uint32_t* cur, uint32_t* next, const uint32_t* counter) {
    next[0] = cur[1];
    next[1] = *counter;
}

// Closest hit through the wide BVH: the hit children of a node in order of
// entry distance; leaf children's triangles tested at once, internal ones
// pushed (with their entry distance, so that a popped node already beyond
// the closest hit is skipped). Same triangle test and tie rule as the binary
// traversal, and conservative boxes, so the same hits as brute force.
__global__ void __launch_bounds__(128) trace_wide_kernel(const WNode* __restrict__ wn,
                                                         const TriRec* __restrict__ tris,
                                                         const float4* __restrict__ rays, uint32_t n_rays,
                                                         float* __restrict__ hit_t,
                                                         uint32_t* __restrict__ hit_prim, Counts* counts,
                                                         int* err, const uint32_t* __restrict__ order) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t c_nodes = 0, c_boxes = 0, c_tris = 0;
    if (j < n_rays) {
        const uint32_t i = order ? order[j] : j;  // the ray this thread traces
        const float4 o = rays[2 * i], d = rays[2 * i + 1];
        const float ix = __fdiv_rn(1.0f, d.x), iy = __fdiv_rn(1.0f, d.y), iz = __fdiv_rn(1.0f, d.z);
        float best = __int_as_float(0x7F800000);
        uint32_t best_prim = kNoHit;
        uint32_t st_node[kWideStack];
        float st_t[kWideStack];
        int sp = 0;
        st_node[sp] = 0;
        st_t[sp] = 0.0f;
        ++sp;
        bool overflow = false;
        while (sp > 0) {
            --sp;
            if (st_t[sp] > best) continue;
            const uint32_t ni = st_node[sp];
            c_nodes++;
            const float4* q4 = reinterpret_cast<const float4*>(wn + ni);
            const float4 h0 = q4[0], h1 = q4[1], h2 = q4[2], h3 = q4[3], h4 = q4[4], h5 = q4[5], h6 = q4[6];
            const uint32_t ew = __float_as_uint(h0.w);
            const float sx = wstep(ew & 0xFFu), sy = wstep((ew >> 8) & 0xFFu), sz = wstep((ew >> 16) & 0xFFu);
            const uint32_t m = ew >> 24;
            const uint32_t ql[3][2] = {{__float_as_uint(h1.x), __float_as_uint(h1.y)},
                                       {__float_as_uint(h1.z), __float_as_uint(h1.w)},
                                       {__float_as_uint(h2.x), __float_as_uint(h2.y)}};
            const uint32_t qh[3][2] = {{__float_as_uint(h2.z), __float_as_uint(h2.w)},
                                       {__float_as_uint(h3.x), __float_as_uint(h3.y)},
                                       {__float_as_uint(h3.z), __float_as_uint(h3.w)}};
            const uint32_t refs[8] = {__float_as_uint(h4.x), __float_as_uint(h4.y), __float_as_uint(h4.z),
                                      __float_as_uint(h4.w), __float_as_uint(h5.x), __float_as_uint(h5.y),
                                      __float_as_uint(h5.z), __float_as_uint(h5.w)};
            const uint32_t cnt2[2] = {__float_as_uint(h6.x), __float_as_uint(h6.y)};
            float ent[8];
            uint32_t hitm = 0, leafm = 0;
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) {
                ent[j] = __int_as_float(0x7FFFFFFF);
                if (j < m) {
                    const uint32_t sh = (j & 3u) * 8u, wd = j >> 2;
                    const float4 lo = make_float4(wdeq(h0.x, (ql[0][wd] >> sh) & 0xFFu, sx),
                                                  wdeq(h0.y, (ql[1][wd] >> sh) & 0xFFu, sy),
                                                  wdeq(h0.z, (ql[2][wd] >> sh) & 0xFFu, sz), 0.0f);
                    const float4 hi = make_float4(wdeq(h0.x, (qh[0][wd] >> sh) & 0xFFu, sx),
                                                  wdeq(h0.y, (qh[1][wd] >> sh) & 0xFFu, sy),
                                                  wdeq(h0.z, (qh[2][wd] >> sh) & 0xFFu, sz), 0.0f);
                    c_boxes++;
                    ent[j] = box_entry(o.x, o.y, o.z, ix, iy, iz, lo, hi, best);
                    if (ent[j] <= best) hitm |= 1u << j;
                    if (refs[j] & kWideLeaf) leafm |= 1u << j;
                }
            }
            // leaf children, nearest first (selections over a bit mask: no
            // indexed arrays, everything stays in registers)
            uint32_t lm = hitm & leafm;
            while (lm) {
                float be = __int_as_float(0x7F800000);
                uint32_t bj = 0, br = 0, bc = 0;
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j)
                    if (((lm >> j) & 1u) && !(ent[j] >= be)) {
                        be = ent[j];
                        bj = j;
                        br = refs[j];
                        bc = (cnt2[j >> 2] >> ((j & 3u) * 8u)) & 0xFFu;
                    }
                lm &= ~(1u << bj);
                if (be > best) continue;
                const uint32_t start = br & ~kWideLeaf;
                for (uint32_t q = start; q < start + bc; ++q) {
                    const TriRec t = tris[q];
                    c_tris++;
                    const float tt = intersect_tri(o.x, o.y, o.z, d.x, d.y, d.z, t);
                    const uint32_t prim = __float_as_uint(t.a.w);
                    if (tt >= 0.0f && (tt < best || (tt == best && prim < best_prim))) {
                        best = tt;
                        best_prim = prim;
                    }
                }
            }
            // internal children pushed farthest first (popped nearest first)
            uint32_t im = hitm & ~leafm;
            while (im) {
                float be = -1.0f;
                uint32_t bj = 0, br = 0;
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j)
                    if (((im >> j) & 1u) && ent[j] >= be) {
                        be = ent[j];
                        bj = j;
                        br = refs[j];
                    }
                im &= ~(1u << bj);
                if (be > best) continue;
                if (sp >= kWideStack) {
                    overflow = true;
                    break;
                }
                st_node[sp] = br;
                st_t[sp] = be;
                ++sp;
            }
            if (overflow) {
                atomicExch(err, 1);
                break;
            }
        }
        hit_t[i] = best_prim == kNoHit ? -1.0f : best;
        hit_prim[i] = best_prim;
    }
    if (counts) {
        unsigned long long a = c_nodes, b = c_boxes, c = c_tris;
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_down_sync(kFull, a, off);
            b += __shfl_down_sync(kFull, b, off);
            c += __shfl_down_sync(kFull, c, off);
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicAdd(&counts->nodes, a);
            atomicAdd(&counts->boxes, b);
            atomicAdd(&counts->tris, c);
        }
    }
}


// trace_wide_kernel with persistent warps that refill idle lanes
// (trace_persistent_kernel's scheme): the same node steps, tests and results.
__global__ void __launch_bounds__(128) trace_wide_persistent_kernel(
    const WNode* __restrict__ wn, const TriRec* __restrict__ tris, const float4* __restrict__ rays,
    uint32_t n_rays, float* __restrict__ hit_t, uint32_t* __restrict__ hit_prim, Counts* counts, int* err,
    const uint32_t* __restrict__ order, uint32_t* __restrict__ next) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t c_nodes = 0, c_boxes = 0, c_tris = 0;
    bool has = false, exhausted = false;
    uint32_t ri = 0, best_prim = kNoHit;
    float ox = 0.f, oy = 0.f, oz = 0.f, dx = 0.f, dy = 0.f, dz = 0.f, ix = 0.f, iy = 0.f, iz = 0.f;
    float best = 0.f;
    uint32_t st_node[kWideStack];
    float st_t[kWideStack];
    int sp = 0;
    for (;;) {
        const uint32_t idle = __ballot_sync(kFull, !has);
        if (!exhausted && idle != 0u &&
            (static_cast<uint32_t>(__popc(idle)) >= MGBVH_TRACE_REFILL || idle == kFull)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(next, static_cast<uint32_t>(__popc(idle)));
            base = __shfl_sync(kFull, base, 0);
            if (base >= n_rays) exhausted = true;  // warp-uniform
            if (!has) {
                const uint32_t jr = base + static_cast<uint32_t>(__popc(idle & ((1u << lane) - 1u)));
                if (jr < n_rays) {
                    ri = order ? order[jr] : jr;
                    const float4 o = rays[2 * ri], d = rays[2 * ri + 1];
                    ox = o.x, oy = o.y, oz = o.z, dx = d.x, dy = d.y, dz = d.z;
                    ix = __fdiv_rn(1.0f, d.x), iy = __fdiv_rn(1.0f, d.y), iz = __fdiv_rn(1.0f, d.z);
                    best = __int_as_float(0x7F800000);
                    best_prim = kNoHit;
                    st_node[0] = 0;
                    st_t[0] = 0.0f;
                    sp = 1;
                    has = true;
                }
            }
        }
        if (!__any_sync(kFull, has)) {
            if (exhausted) break;
            continue;  // all lanes idle: the loop's next pass refills them
        }
        if (has && sp > 0) {
            --sp;
            if (!(st_t[sp] > best)) {
                bool overflow = false;
                    const uint32_t ni = st_node[sp];
                    c_nodes++;
                    const float4* q4 = reinterpret_cast<const float4*>(wn + ni);
                    const float4 h0 = q4[0], h1 = q4[1], h2 = q4[2], h3 = q4[3], h4 = q4[4], h5 = q4[5], h6 = q4[6];
                    const uint32_t ew = __float_as_uint(h0.w);
                    const float sx = wstep(ew & 0xFFu), sy = wstep((ew >> 8) & 0xFFu), sz = wstep((ew >> 16) & 0xFFu);
                    const uint32_t m = ew >> 24;
                    const uint32_t ql[3][2] = {{__float_as_uint(h1.x), __float_as_uint(h1.y)},
                                               {__float_as_uint(h1.z), __float_as_uint(h1.w)},
                                               {__float_as_uint(h2.x), __float_as_uint(h2.y)}};
                    const uint32_t qh[3][2] = {{__float_as_uint(h2.z), __float_as_uint(h2.w)},
                                               {__float_as_uint(h3.x), __float_as_uint(h3.y)},
                                               {__float_as_uint(h3.z), __float_as_uint(h3.w)}};
                    const uint32_t refs[8] = {__float_as_uint(h4.x), __float_as_uint(h4.y), __float_as_uint(h4.z),
                                              __float_as_uint(h4.w), __float_as_uint(h5.x), __float_as_uint(h5.y),
                                              __float_as_uint(h5.z), __float_as_uint(h5.w)};
                    const uint32_t cnt2[2] = {__float_as_uint(h6.x), __float_as_uint(h6.y)};
                    float ent[8];
                    uint32_t hitm = 0, leafm = 0;
        #pragma unroll
                    for (uint32_t j = 0; j < 8; ++j) {
                        ent[j] = __int_as_float(0x7FFFFFFF);
                        if (j < m) {
                            const uint32_t sh = (j & 3u) * 8u, wd = j >> 2;
                            const float4 lo = make_float4(wdeq(h0.x, (ql[0][wd] >> sh) & 0xFFu, sx),
                                                          wdeq(h0.y, (ql[1][wd] >> sh) & 0xFFu, sy),
                                                          wdeq(h0.z, (ql[2][wd] >> sh) & 0xFFu, sz), 0.0f);
                            const float4 hi = make_float4(wdeq(h0.x, (qh[0][wd] >> sh) & 0xFFu, sx),
                                                          wdeq(h0.y, (qh[1][wd] >> sh) & 0xFFu, sy),
                                                          wdeq(h0.z, (qh[2][wd] >> sh) & 0xFFu, sz), 0.0f);
                            c_boxes++;
                            ent[j] = box_entry(ox, oy, oz, ix, iy, iz, lo, hi, best);
                            if (ent[j] <= best) hitm |= 1u << j;
                            if (refs[j] & kWideLeaf) leafm |= 1u << j;
                        }
                    }
                    // leaf children, nearest first (selections over a bit mask: no
                    // indexed arrays, everything stays in registers)
                    uint32_t lm = hitm & leafm;
                    while (lm) {
                        float be = __int_as_float(0x7F800000);
                        uint32_t bj = 0, br = 0, bc = 0;
        #pragma unroll
                        for (uint32_t j = 0; j < 8; ++j)
                            if (((lm >> j) & 1u) && !(ent[j] >= be)) {
                                be = ent[j];
                                bj = j;
                                br = refs[j];
                                bc = (cnt2[j >> 2] >> ((j & 3u) * 8u)) & 0xFFu;
                            }
                        lm &= ~(1u << bj);
                        if (be > best) continue;
                        const uint32_t start = br & ~kWideLeaf;
                        for (uint32_t q = start; q < start + bc; ++q) {
                            const TriRec t = tris[q];
                            c_tris++;
                            const float tt = intersect_tri(ox, oy, oz, dx, dy, dz, t);
                            const uint32_t prim = __float_as_uint(t.a.w);
                            if (tt >= 0.0f && (tt < best || (tt == best && prim < best_prim))) {
                                best = tt;
                                best_prim = prim;
                            }
                        }
                    }
                    // internal children pushed farthest first (popped nearest first)
                    uint32_t im = hitm & ~leafm;
                    while (im) {
                        float be = -1.0f;
                        uint32_t bj = 0, br = 0;
        #pragma unroll
                        for (uint32_t j = 0; j < 8; ++j)
                            if (((im >> j) & 1u) && ent[j] >= be) {
                                be = ent[j];
                                bj = j;
                                br = refs[j];
                            }
                        im &= ~(1u << bj);
                        if (be > best) continue;
                        if (sp >= kWideStack) {
                            overflow = true;
                            break;
                        }
                        st_node[sp] = br;
                        st_t[sp] = be;
                        ++sp;
                    }
                if (overflow) {
                    atomicExch(err, 1);
                    sp = 0;
                }
            }
        }
        if (has && sp == 0) {
            hit_t[ri] = best_prim == kNoHit ? -1.0f : best;
            hit_prim[ri] = best_prim;
            has = false;
        }
    }
    if (counts) {
        unsigned long long a = c_nodes, b = c_boxes, c = c_tris;
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_down_sync(kFull, a, off);
            b += __shfl_down_sync(kFull, b, off);
            c += __shfl_down_sync(kFull, c, off);
        }
        if (lane == 0) {
            atomicAdd(&counts->nodes, a);
            atomicAdd(&counts->boxes, b);
            atomicAdd(&counts->tris, c);
        }
    }
}

// Ray order per traversal (tuning knobs): 0 as given, 1 direction bin then
// origin, 2 origin cell then direction bin. Measured on 8.4M random rays in a
// 16.8M-triangle scene: binary 34.2 / 44.6 / 49.3 Mrays/s, 8-wide 28.9 /
// 39.3 / 37.2 Mrays/s for 0 / 1 / 2 (form 2 at 256 cells per axis and 4
// bins per component); form 2 with 16 cells and 8 bins: binary 54.5,
// 8-wide 41.9.
#ifndef MGBVH_RAY_SORT_BINARY
#define MGBVH_RAY_SORT_BINARY 2
#endif
#ifndef MGBVH_RAY_SORT_WIDE
#define MGBVH_RAY_SORT_WIDE 2
#endif

// Sort key of a ray for the tracing order. Mode 1: the direction quantized
// to 4 bins per component (6 bits) above the origin quantized to 256 cells
// per axis of the root box, Morton-interleaved (24 bits). Mode 2: the origin
// cell at 2^MGBVH_RAY_ORIGIN_BITS per axis (Morton) above the direction at
// 2^MGBVH_RAY_DIR_BITS bins per component. Rays that start near one another
// in similar directions then share warps. The order changes no hit.
__device__ __forceinline__ uint32_t spread8(uint32_t v) {  // 8 bits -> every third of 24
    v &= 0xFFu;
    v = (v | (v << 8)) & 0x00F00Fu;
    v = (v | (v << 4)) & 0x0C30C3u;
    v = (v | (v << 2)) & 0x249249u;
    return v;
}

#ifndef MGBVH_RAY_ORIGIN_BITS
#define MGBVH_RAY_ORIGIN_BITS 4  // origin-first key: origin cells per axis = 2^bits (tuning knob)
#endif
#ifndef MGBVH_RAY_DIR_BITS
#define MGBVH_RAY_DIR_BITS 3  // origin-first key: direction bins per component = 2^bits (tuning knob)
#endif
constexpr uint32_t kRayKeyBits2 = 3u * (MGBVH_RAY_ORIGIN_BITS + MGBVH_RAY_DIR_BITS);
static_assert(kRayKeyBits2 <= 30u, "ray key wider than 30 bits");

__global__ void ray_key_kernel(const float4* __restrict__ rays, uint32_t n, const float4* __restrict__ root,
                               uint32_t mode, uint32_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const float4 lo = root[0], hi = root[1];
    const float sx = 256.0f / fmaxf(hi.x - lo.x, 1e-30f), sy = 256.0f / fmaxf(hi.y - lo.y, 1e-30f),
                sz = 256.0f / fmaxf(hi.z - lo.z, 1e-30f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = rays[2 * i], d = rays[2 * i + 1];
        const uint32_t qx = (uint32_t)fminf(fmaxf((o.x - lo.x) * sx, 0.0f), 255.0f);
        const uint32_t qy = (uint32_t)fminf(fmaxf((o.y - lo.y) * sy, 0.0f), 255.0f);
        const uint32_t qz = (uint32_t)fminf(fmaxf((o.z - lo.z) * sz, 0.0f), 255.0f);
        const uint32_t morton = spread8(qx) | (spread8(qy) << 1) | (spread8(qz) << 2);
        const uint32_t dx = (uint32_t)fminf(fmaxf((d.x + 1.0f) * 2.0f, 0.0f), 3.0f);
        const uint32_t dy = (uint32_t)fminf(fmaxf((d.y + 1.0f) * 2.0f, 0.0f), 3.0f);
        const uint32_t dz = (uint32_t)fminf(fmaxf((d.z + 1.0f) * 2.0f, 0.0f), 3.0f);
        const uint32_t dir = dx | (dy << 2) | (dz << 4);
        if (mode == 1) {
            keys[i] = (dir << 24) | morton;
        } else {
            // origin first at MGBVH_RAY_ORIGIN_BITS per axis, then the direction
            // at MGBVH_RAY_DIR_BITS per component
            constexpr uint32_t ob = MGBVH_RAY_ORIGIN_BITS, db = MGBVH_RAY_DIR_BITS;
            const uint32_t m2 = morton >> (3u * (8u - ob));
            const float nd = (float)(1u << db);
            const uint32_t ex = (uint32_t)fminf(fmaxf((d.x + 1.0f) * 0.5f * nd, 0.0f), nd - 1.0f);
            const uint32_t ey = (uint32_t)fminf(fmaxf((d.y + 1.0f) * 0.5f * nd, 0.0f), nd - 1.0f);
            const uint32_t ez = (uint32_t)fminf(fmaxf((d.z + 1.0f) * 0.5f * nd, 0.0f), nd - 1.0f);
            keys[i] = (m2 << (3u * db)) | ex | (ey << db) | (ez << (2u * db));
        }
        idx[i] = i;
    }
}

// ---------------------------------------------------------------- two-level scenes
//
// The reference's scene traversal (scene.slang:91-141 raytraceTlas, :143-220
// raytraceBlas): the TLAS is walked with the world ray; at a TLAS leaf the
// ray moves into the instance's mesh space through its inverse transform
// (:161-164) and that mesh's BLAS is walked from its root (:172), on the same
// stack. The hit distance stays the world ray's parameter: the mesh-space ray
// o' = M o, d' = M d (d' not normalized) reaches M p at the same t as the
// world ray reaches p, so distances compare across instances as they are
// (the shader's rescaling by |d'|, :168-169, is wrong for scaled instances
// and is not copied). Equal distances resolve to the lowest (instance,
// triangle) pair, and TLAS boxes are tested grown by a relative 1e-5 (they
// come from f32 corner transforms, which can round a hair inside the exact
// transformed mesh), so the traversal finds exactly the brute-force hits.

struct SceneMesh {  // mgbvh_scene_mesh
    uint32_t blas_root, tri_offset, tri_count, vertex_offset;
};

struct SceneInst {  // mgbvh_scene_instance
    float m[16];  // column-major world -> mesh
    uint32_t mesh, pad[3];
};

constexpr int kSceneStack = 96;  // a TLAS path and a BLAS path of up to 47 levels each

// Column-major M * (x, y, z, w), each component ((c0 x + c1 y) + c2 z) + c3 w
// with every product and sum rounded (glam's f32 Mat4 * Vec4 order).
__device__ __forceinline__ void xform(const float* m, float x, float y, float z, float w, float& ox, float& oy,
                                      float& oz) {
    ox = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], x), __fmul_rn(m[4], y)), __fmul_rn(m[8], z)),
                   __fmul_rn(m[12], w));
    oy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[1], x), __fmul_rn(m[5], y)), __fmul_rn(m[9], z)),
                   __fmul_rn(m[13], w));
    oz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[2], x), __fmul_rn(m[6], y)), __fmul_rn(m[10], z)),
                   __fmul_rn(m[14], w));
}

__device__ __forceinline__ float4 grow_lo(float4 v) {
    return make_float4(v.x - fabsf(v.x) * 1e-5f - 1e-30f, v.y - fabsf(v.y) * 1e-5f - 1e-30f,
                       v.z - fabsf(v.z) * 1e-5f - 1e-30f, v.w);
}
__device__ __forceinline__ float4 grow_hi(float4 v) {
    return make_float4(v.x + fabsf(v.x) * 1e-5f + 1e-30f, v.y + fabsf(v.y) * 1e-5f + 1e-30f,
                       v.z + fabsf(v.z) * 1e-5f + 1e-30f, v.w);
}

// (t, instance, triangle) strictly before the current best.
__device__ __forceinline__ bool scene_better(float tt, uint32_t inst, uint32_t tri, float best, uint32_t bi,
                                             uint32_t bp) {
    return tt < best || (tt == best && (inst < bi || (inst == bi && tri < bp)));
}

template <bool kTlasLens, bool kBlasLens>
__global__ void __launch_bounds__(128) trace_scene_kernel(
    const float4* __restrict__ tlas, const uint32_t* __restrict__ tlas_lens, const SceneInst* __restrict__ inst,
    uint32_t n_inst, const SceneMesh* __restrict__ meshes, uint32_t n_meshes, const float4* __restrict__ blas,
    const uint32_t* __restrict__ blas_lens, const TriRec* __restrict__ tris, const float4* __restrict__ rays,
    uint32_t n_rays, float* __restrict__ hit_t, uint32_t* __restrict__ hit_inst, uint32_t* __restrict__ hit_tri,
    Counts* counts, int* err, const uint32_t* __restrict__ order) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t c_nodes = 0, c_boxes = 0, c_tris = 0;
    if (j < n_rays) {
        const uint32_t i = order ? order[j] : j;
        const float4 o = rays[2 * i], d = rays[2 * i + 1];
        const float ix = __fdiv_rn(1.0f, d.x), iy = __fdiv_rn(1.0f, d.y), iz = __fdiv_rn(1.0f, d.z);
        float best = __int_as_float(0x7F800000);
        uint32_t bi = kNoHit, bp = kNoHit;
        uint32_t stack[kSceneStack];
        int sp = 0;
        c_boxes++;
        if (box_entry(o.x, o.y, o.z, ix, iy, iz, grow_lo(tlas[0]), grow_hi(tlas[1]), best) <= best) stack[sp++] = 0;
        while (sp > 0) {
            const uint32_t ni = stack[--sp];
            c_nodes++;
            const float4 nhi = tlas[2 * ni + 1];
            const uint32_t child = __float_as_uint(nhi.w);
            if (child != 0) {
                c_boxes += 2;
                const float da = box_entry(o.x, o.y, o.z, ix, iy, iz, grow_lo(tlas[2 * child]),
                                           grow_hi(tlas[2 * child + 1]), best);
                const float db = box_entry(o.x, o.y, o.z, ix, iy, iz, grow_lo(tlas[2 * child + 2]),
                                           grow_hi(tlas[2 * child + 3]), best);
                const bool pa = da <= best, pb = db <= best;
                if (sp + 2 > kSceneStack) {
                    atomicExch(err, 1);
                    break;
                }
                if (pa && pb) {
                    const bool a_first = da < db;
                    stack[sp++] = a_first ? child + 1 : child;
                    stack[sp++] = a_first ? child : child + 1;
                } else if (pa || pb) {
                    stack[sp++] = pa ? child : child + 1;
                }
                continue;
            }
            const uint32_t start = __float_as_uint(tlas[2 * ni].w);
            const uint32_t len = kTlasLens ? tlas_lens[ni] : 1u;
            for (uint32_t k = start; k < start + len; ++k) {
                if (k >= n_inst || inst[k].mesh >= n_meshes) {
                    atomicExch(err, 2);
                    continue;
                }
                const SceneInst& I = inst[k];
                const SceneMesh M = meshes[I.mesh];
                if (M.tri_count == 0) continue;  // an empty mesh: no BLAS
                float lox, loy, loz, ldx, ldy, ldz;
                xform(I.m, o.x, o.y, o.z, 1.0f, lox, loy, loz);
                xform(I.m, d.x, d.y, d.z, 0.0f, ldx, ldy, ldz);
                const float lix = __fdiv_rn(1.0f, ldx), liy = __fdiv_rn(1.0f, ldy), liz = __fdiv_rn(1.0f, ldz);
                const float4* bn = blas + 2 * (size_t)M.blas_root;
                const uint32_t* bl = kBlasLens ? blas_lens + M.blas_root : nullptr;
                // the mesh's BLAS on the same stack, from its root (scene.slang:171-173)
                const int base = sp;
                if (sp + 1 > kSceneStack) {
                    atomicExch(err, 1);
                    break;
                }
                stack[sp++] = 0;
                while (sp > base) {
                    const uint32_t bi_ = stack[--sp];
                    c_nodes++;
                    const uint32_t bchild = __float_as_uint(bn[2 * bi_ + 1].w);
                    if (bchild != 0) {
                        c_boxes += 2;
                        const float da = box_entry(lox, loy, loz, lix, liy, liz, bn[2 * bchild], bn[2 * bchild + 1], best);
                        const float db =
                            box_entry(lox, loy, loz, lix, liy, liz, bn[2 * bchild + 2], bn[2 * bchild + 3], best);
                        const bool pa = da <= best, pb = db <= best;
                        if (sp + 2 > kSceneStack) {
                            atomicExch(err, 1);
                            sp = base;
                            break;
                        }
                        if (pa && pb) {
                            const bool a_first = da < db;
                            stack[sp++] = a_first ? bchild + 1 : bchild;
                            stack[sp++] = a_first ? bchild : bchild + 1;
                        } else if (pa || pb) {
                            stack[sp++] = pa ? bchild : bchild + 1;
                        }
                    } else {
                        const uint32_t s0 = __float_as_uint(bn[2 * bi_].w);
                        const uint32_t n0 = kBlasLens ? bl[bi_] : 1u;
                        for (uint32_t q = s0; q < s0 + n0 && q < M.tri_count; ++q) {
                            const uint32_t tri = M.tri_offset + q;
                            c_tris++;
                            const float tt = intersect_tri(lox, loy, loz, ldx, ldy, ldz, tris[tri]);
                            if (tt >= 0.0f && scene_better(tt, k, tri, best, bi, bp)) {
                                best = tt;
                                bi = k;
                                bp = tri;
                            }
                        }
                    }
                }
            }
        }
        hit_t[i] = bp == kNoHit ? -1.0f : best;
        hit_inst[i] = bi;
        hit_tri[i] = bp;
    }
    if (counts) {
        unsigned long long a = c_nodes, b = c_boxes, c = c_tris;
        for (int off = 16; off > 0; off >>= 1) {
            a += __shfl_down_sync(kFull, a, off);
            b += __shfl_down_sync(kFull, b, off);
            c += __shfl_down_sync(kFull, c, off);
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicAdd(&counts->nodes, a);
            atomicAdd(&counts->boxes, b);
            atomicAdd(&counts->tris, c);
        }
    }
}

// Brute force over a scene: one CTA per ray; for every instance the ray in
// mesh space, then every triangle of the mesh (threads split the triangles).
// cull != 0 skips an instance whose mesh-space ray misses the mesh's BLAS
// root box grown by a relative 1e-4 (a filter far wider than any rounding;
// it keeps large scenes affordable).
constexpr int kBruteThreads = 256;

__global__ void __launch_bounds__(kBruteThreads) brute_scene_kernel(
    const SceneInst* __restrict__ inst, uint32_t n_inst, const SceneMesh* __restrict__ meshes, uint32_t n_meshes,
    const float4* __restrict__ blas, const TriRec* __restrict__ tris, const float4* __restrict__ rays,
    uint32_t n_rays, float* __restrict__ hit_t, uint32_t* __restrict__ hit_inst, uint32_t* __restrict__ hit_tri,
    int cull) {
    __shared__ float st[kBruteThreads];
    __shared__ uint32_t si[kBruteThreads], sp[kBruteThreads];
    for (uint32_t r = blockIdx.x; r < n_rays; r += gridDim.x) {
        const float4 o = rays[2 * r], d = rays[2 * r + 1];
        float best = __int_as_float(0x7F800000);
        uint32_t bi = kNoHit, bp = kNoHit;
        for (uint32_t k = 0; k < n_inst; ++k) {
            const SceneInst& I = inst[k];
            if (I.mesh >= n_meshes) continue;
            const SceneMesh M = meshes[I.mesh];
            if (M.tri_count == 0) continue;
            float lox, loy, loz, ldx, ldy, ldz;
            xform(I.m, o.x, o.y, o.z, 1.0f, lox, loy, loz);
            xform(I.m, d.x, d.y, d.z, 0.0f, ldx, ldy, ldz);
            if (cull) {
                float4 lo = blas[2 * (size_t)M.blas_root], hi = blas[2 * (size_t)M.blas_root + 1];
                const float gx = (fabsf(lo.x) + fabsf(hi.x)) * 1e-4f + 1e-30f;
                const float gy = (fabsf(lo.y) + fabsf(hi.y)) * 1e-4f + 1e-30f;
                const float gz = (fabsf(lo.z) + fabsf(hi.z)) * 1e-4f + 1e-30f;
                lo = make_float4(lo.x - gx, lo.y - gy, lo.z - gz, 0.f);
                hi = make_float4(hi.x + gx, hi.y + gy, hi.z + gz, 0.f);
                const float lix = __fdiv_rn(1.0f, ldx), liy = __fdiv_rn(1.0f, ldy), liz = __fdiv_rn(1.0f, ldz);
                if (!(box_entry(lox, loy, loz, lix, liy, liz, lo, hi, __int_as_float(0x7F800000)) >= 0.0f))
                    continue;  // block-uniform
            }
            for (uint32_t q = threadIdx.x; q < M.tri_count; q += blockDim.x) {
                const uint32_t tri = M.tri_offset + q;
                const float tt = intersect_tri(lox, loy, loz, ldx, ldy, ldz, tris[tri]);
                if (tt >= 0.0f && scene_better(tt, k, tri, best, bi, bp)) {
                    best = tt;
                    bi = k;
                    bp = tri;
                }
            }
        }
        st[threadIdx.x] = best;
        si[threadIdx.x] = bi;
        sp[threadIdx.x] = bp;
        __syncthreads();
        for (int s = kBruteThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < (uint32_t)s) {
                const uint32_t o2 = threadIdx.x + s;
                if (sp[o2] != kNoHit &&
                    (sp[threadIdx.x] == kNoHit || scene_better(st[o2], si[o2], sp[o2], st[threadIdx.x],
                                                               si[threadIdx.x], sp[threadIdx.x]))) {
                    st[threadIdx.x] = st[o2];
                    si[threadIdx.x] = si[o2];
                    sp[threadIdx.x] = sp[o2];
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            hit_t[r] = sp[0] == kNoHit ? -1.0f : st[0];
            hit_inst[r] = si[0];
            hit_tri[r] = sp[0];
        }
        __syncthreads();
    }
}

// The scene's triangles with their vertices, mesh by mesh (blockIdx.y):
// TriRec k holds triangle k of the scene array (indices relative to its
// mesh's vertex offset), id = k.
__global__ void gather_scene_kernel(const float* __restrict__ verts, uint32_t stride_floats, uint32_t nverts,
                                    const uint32_t* __restrict__ tris, uint32_t n_tris,
                                    const SceneMesh* __restrict__ meshes, TriRec* __restrict__ out, int* err) {
    const SceneMesh M = meshes[blockIdx.y];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < M.tri_count; q += gridDim.x * blockDim.x) {
        const uint32_t k = M.tri_offset + q;
        if (k >= n_tris) {
            atomicExch(err, 2);
            continue;
        }
        uint32_t v[3];
        bool bad = false;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            v[c] = tris[3 * (size_t)k + c] + M.vertex_offset;
            bad |= v[c] >= nverts || v[c] < M.vertex_offset;
        }
        if (bad) {
            atomicExch(err, 2);
            continue;
        }
        const float* a = verts + (size_t)v[0] * stride_floats;
        const float* b = verts + (size_t)v[1] * stride_floats;
        const float* c = verts + (size_t)v[2] * stride_floats;
        TriRec r;
        r.a = make_float4(a[0], a[1], a[2], __uint_as_float(k));
        r.b = make_float4(b[0], b[1], b[2], 0.0f);
        r.c = make_float4(c[0], c[1], c[2], 0.0f);
        out[k] = r;
    }
}

}  // namespace mgbvh_trace

using namespace mgbvh_trace;

struct mgbvh_tracer {
    int device = 0;
    TriRec* tris = nullptr;
    size_t tris_cap = 0;
    uint32_t n_tris = 0;
    const mgbvh_node* nodes = nullptr;
    const uint32_t* lens = nullptr;
    uint32_t node_count = 0;
    Counts* d_counts = nullptr;
    int* d_err = nullptr;
    uint32_t* d_next = nullptr;  // persistent traversal: next ray to hand out
    int trace_blocks = 0;        // persistent traversal: resident CTAs of 128 threads
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.0f;
    // the wide BVH of the bound tree (mgbvh_tracer_build_wide)
    WNode* wide = nullptr;
    uint32_t* wbin = nullptr;
    uint32_t* wlen = nullptr;
    uint32_t* wmeta = nullptr;  // [0..1], [2..3]: level ranges; [4]: slots taken
    size_t wide_cap = 0;
    uint32_t wide_count = 0;
    // tracing order: ray keys and indices (two of each for the radix sort)
    uint32_t* rkey[2] = {nullptr, nullptr};
    uint32_t* ridx[2] = {nullptr, nullptr};
    size_t ray_cap = 0;
    void* sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    // a two-level scene (mgbvh_tracer_set_scene_dev): the caller's TLAS,
    // instances and BLAS nodes (kept as pointers), the mesh table (copied)
    bool scene = false;
    const mgbvh_node* tlas = nullptr;
    const uint32_t* tlas_lens = nullptr;
    const SceneInst* inst = nullptr;
    uint32_t n_inst = 0;
    SceneMesh* meshes = nullptr;
    size_t meshes_cap = 0;
    uint32_t n_meshes = 0;
    const mgbvh_node* blas = nullptr;
    const uint32_t* blas_lens = nullptr;
};

namespace {

int trace_check(cudaError_t e) { return e == cudaSuccess ? MGBVH_OK : MGBVH_ERR_CUDA; }

// Buffers of the tracing order for n rays (grown before the timed region).
int ensure_order_buffers(mgbvh_tracer* t, uint32_t n) {
    if (t->ray_cap < n) {
        for (int k = 0; k < 2; ++k) {
            if (t->rkey[k]) cudaFree(t->rkey[k]);
            if (t->ridx[k]) cudaFree(t->ridx[k]);
            t->rkey[k] = t->ridx[k] = nullptr;
        }
        t->ray_cap = 0;
        for (int k = 0; k < 2; ++k)
            if (cudaMalloc(&t->rkey[k], 4ull * n) != cudaSuccess || cudaMalloc(&t->ridx[k], 4ull * n) != cudaSuccess)
                return MGBVH_ERR_CUDA;
        t->ray_cap = n;
    }
    size_t need = 0;
    cub::DoubleBuffer<uint32_t> kb(t->rkey[0], t->rkey[1]), vb(t->ridx[0], t->ridx[1]);
    if (cub::DeviceRadixSort::SortPairs(nullptr, need, kb, vb, (int)n, 0, 30) != cudaSuccess) return MGBVH_ERR_CUDA;
    if (t->sort_tmp_bytes < need) {
        if (t->sort_tmp) cudaFree(t->sort_tmp);
        t->sort_tmp = nullptr;
        t->sort_tmp_bytes = 0;
        if (cudaMalloc(&t->sort_tmp, need) != cudaSuccess) return MGBVH_ERR_CUDA;
        t->sort_tmp_bytes = need;
    }
    return MGBVH_OK;
}

// Enqueues the tracing order of the rays on stream sm: keys (ray_key_kernel
// mode), then a radix sort of (key, ray index); returns the sorted ray
// indices, or nullptr (rays traced as given).
const uint32_t* ray_order(mgbvh_tracer* t, const float4* rays, uint32_t n, cudaStream_t sm, uint32_t mode,
                          const mgbvh_node* root = nullptr) {
    if (mode == 0) return nullptr;
    ray_key_kernel<<<1184, 256, 0, sm>>>(rays, n, reinterpret_cast<const float4*>(root ? root : t->nodes), mode,
                                         t->rkey[0], t->ridx[0]);
    cub::DoubleBuffer<uint32_t> kb(t->rkey[0], t->rkey[1]), vb(t->ridx[0], t->ridx[1]);
    size_t bytes = t->sort_tmp_bytes;
    if (cub::DeviceRadixSort::SortPairs(t->sort_tmp, bytes, kb, vb, (int)n, 0, 30, sm) != cudaSuccess)
        return nullptr;
    return vb.Current();
}

}  // namespace

extern "C" {

int mgbvh_tracer_create(int device, mgbvh_tracer** out) {
    if (!out) return MGBVH_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return MGBVH_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev || cudaSetDevice(device) != cudaSuccess) return MGBVH_ERR_INVALID_ARG;
    mgbvh_tracer* t = new mgbvh_tracer();
    t->device = device;
    int sms = 0, per_sm = 0;
    if (cudaMalloc(&t->d_counts, sizeof(Counts)) != cudaSuccess ||
        cudaMalloc(&t->d_err, sizeof(int)) != cudaSuccess || cudaMalloc(&t->d_next, 4) != cudaSuccess ||
        cudaEventCreate(&t->ev0) != cudaSuccess || cudaEventCreate(&t->ev1) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_persistent_kernel<false>, 128, 0) !=
            cudaSuccess) {
        mgbvh_tracer_destroy(t);
        return MGBVH_ERR_CUDA;
    }
    t->trace_blocks = sms * (per_sm > 0 ? per_sm : 1);
    *out = t;
    return MGBVH_OK;
}

void mgbvh_tracer_destroy(mgbvh_tracer* t) {
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->tris) cudaFree(t->tris);
    if (t->wide) cudaFree(t->wide);
    if (t->wbin) cudaFree(t->wbin);
    if (t->wlen) cudaFree(t->wlen);
    if (t->wmeta) cudaFree(t->wmeta);
    if (t->d_counts) cudaFree(t->d_counts);
    if (t->d_err) cudaFree(t->d_err);
    if (t->d_next) cudaFree(t->d_next);
    for (int k = 0; k < 2; ++k) {
        if (t->rkey[k]) cudaFree(t->rkey[k]);
        if (t->ridx[k]) cudaFree(t->ridx[k]);
    }
    if (t->sort_tmp) cudaFree(t->sort_tmp);
    if (t->meshes) cudaFree(t->meshes);
    if (t->ev0) cudaEventDestroy(t->ev0);
    if (t->ev1) cudaEventDestroy(t->ev1);
    delete t;
}

int mgbvh_tracer_set_blas_dev(mgbvh_tracer* t, const mgbvh_node* d_nodes, uint32_t node_count,
                              const uint32_t* d_lens, const float* d_vertices,
                              uint32_t vertex_stride_bytes, uint32_t vertex_count,
                              const uint32_t* d_triangles, const uint32_t* d_perm,
                              uint32_t triangle_count, void* stream) {
    if (!t || !d_nodes || node_count == 0 || !d_vertices || !d_triangles || !d_perm ||
        triangle_count == 0 || vertex_stride_bytes < 12 || vertex_stride_bytes % 4)
        return MGBVH_ERR_INVALID_ARG;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    const size_t need = sizeof(TriRec) * (size_t)triangle_count;
    if (t->tris_cap < need) {
        if (t->tris) cudaFree(t->tris);
        t->tris = nullptr;
        t->tris_cap = 0;
        if (cudaMalloc(&t->tris, need) != cudaSuccess) return MGBVH_ERR_CUDA;
        t->tris_cap = need;
    }
    if (cudaMemsetAsync(t->d_err, 0, sizeof(int), sm) != cudaSuccess) return MGBVH_ERR_CUDA;
    gather_kernel<<<std::max(1u, std::min((triangle_count + 255) / 256, 148u * 16u)), 256, 0, sm>>>(
        d_vertices, vertex_stride_bytes / 4, vertex_count, d_triangles, d_perm, triangle_count,
        t->tris, t->d_err);
    int herr = 0;
    if (cudaMemcpyAsync(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (herr) return MGBVH_ERR_INVALID_ARG;
    t->nodes = d_nodes;
    t->lens = d_lens;
    t->node_count = node_count;
    t->n_tris = triangle_count;
    t->wide_count = 0;  // a wide BVH of an earlier tree no longer applies
    t->scene = false;
    return MGBVH_OK;
}

int mgbvh_tracer_build_wide(mgbvh_tracer* t, void* stream, uint32_t* out_wide_count) {
    if (!t || !t->nodes) return MGBVH_ERR_INVALID_ARG;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    const size_t cap = t->node_count;  // one wide node per internal binary node at most (or the leaf root)
    if (t->wide_cap < cap) {
        if (t->wide) cudaFree(t->wide);
        if (t->wbin) cudaFree(t->wbin);
        if (t->wlen) cudaFree(t->wlen);
        t->wide = nullptr;
        t->wbin = nullptr;
        t->wlen = nullptr;
        t->wide_cap = 0;
        if (cudaMalloc(&t->wide, sizeof(WNode) * cap) != cudaSuccess ||
            cudaMalloc(&t->wbin, sizeof(uint32_t) * cap) != cudaSuccess ||
            cudaMalloc(&t->wlen, sizeof(uint32_t) * cap) != cudaSuccess)
            return MGBVH_ERR_CUDA;
        t->wide_cap = cap;
    }
    if (!t->wmeta && cudaMalloc(&t->wmeta, 8 * sizeof(uint32_t)) != cudaSuccess) return MGBVH_ERR_CUDA;
    const uint32_t init[8] = {0, 1, 0, 0, 1, 0, 0, 0};  // level 0 = [0, 1), one slot taken
    uint32_t hm[8];
    if (cudaMemcpyAsync(t->wmeta, init, sizeof(init), cudaMemcpyHostToDevice, sm) != cudaSuccess ||
        cudaMemsetAsync(t->wbin, 0, sizeof(uint32_t), sm) != cudaSuccess ||  // wide root = binary root
        cudaMemcpyAsync(t->wlen, &t->n_tris, sizeof(uint32_t), cudaMemcpyHostToDevice, sm) != cudaSuccess ||
        cudaMemsetAsync(t->d_err, 0, sizeof(int), sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    const float4* nodes = reinterpret_cast<const float4*>(t->nodes);
    int level = 0;
    bool done = false;
    while (!done) {
        for (int k = 0; k < 8; ++k, ++level) {
            uint32_t* cur = t->wmeta + 2 * (level & 1);
            uint32_t* nxt = t->wmeta + 2 * ((level + 1) & 1);
            wide_level_kernel<<<148 * 8, 128, 0, sm>>>(nodes, t->wbin, t->wlen, cur, t->wmeta + 4, t->wide,
                                                       (uint32_t)cap, t->d_err);
            wide_advance_kernel<<<1, 1, 0, sm>>>(cur, nxt, t->wmeta + 4);
        }
        int herr = 0;
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(hm, t->wmeta, sizeof(hm), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
            cudaMemcpyAsync(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
            cudaStreamSynchronize(sm) != cudaSuccess)
            return MGBVH_ERR_CUDA;
        if (herr) return herr == 4 ? MGBVH_ERR_UNSUPPORTED : MGBVH_ERR_CAPACITY;
        const uint32_t* cur = hm + 2 * (level & 1);
        done = cur[0] == cur[1];
        if (!done && level >= 256) return MGBVH_ERR_CAPACITY;  // deeper than any tree of the builder
    }
    t->wide_count = hm[4];
    if (out_wide_count) *out_wide_count = t->wide_count;
    return MGBVH_OK;
}

int mgbvh_tracer_wide_nodes(mgbvh_tracer* t, const void** d_wide_nodes, uint32_t* wide_count) {
    if (!t || !t->wide_count) return MGBVH_ERR_INVALID_ARG;
    if (d_wide_nodes) *d_wide_nodes = t->wide;
    if (wide_count) *wide_count = t->wide_count;
    return MGBVH_OK;
}

int mgbvh_trace_closest_wide_dev(mgbvh_tracer* t, const float* d_rays, uint32_t n_rays, float* d_hit_t,
                                 uint32_t* d_hit_prim, uint64_t* out_counts, double* out_seconds,
                                 void* stream) {
    if (!t || !t->wide_count || (n_rays && (!d_rays || !d_hit_t || !d_hit_prim))) return MGBVH_ERR_INVALID_ARG;
    if (n_rays == 0) return MGBVH_OK;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(t->d_counts, 0, sizeof(Counts), sm) != cudaSuccess ||
        cudaMemsetAsync(t->d_err, 0, sizeof(int), sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (int rc = ensure_order_buffers(t, n_rays)) return rc;
    cudaEventRecord(t->ev0, sm);
    const float4* rays = reinterpret_cast<const float4*>(d_rays);
    const uint32_t* order = ray_order(t, rays, n_rays, sm, MGBVH_RAY_SORT_WIDE);
    if (MGBVH_TRACE_PERSISTENT) {
        cudaMemsetAsync(t->d_next, 0, 4, sm);
        const int pgrid = (int)std::min<uint32_t>((n_rays + 127) / 128, (uint32_t)t->trace_blocks);
        trace_wide_persistent_kernel<<<pgrid, 128, 0, sm>>>(t->wide, t->tris, rays, n_rays, d_hit_t, d_hit_prim,
                                                            out_counts ? t->d_counts : nullptr, t->d_err, order,
                                                            t->d_next);
    } else {
        trace_wide_kernel<<<(n_rays + 127) / 128, 128, 0, sm>>>(t->wide, t->tris, rays, n_rays, d_hit_t,
                                                                 d_hit_prim, out_counts ? t->d_counts : nullptr,
                                                                 t->d_err, order);
    }
    cudaEventRecord(t->ev1, sm);
    if (cudaGetLastError() != cudaSuccess) return MGBVH_ERR_CUDA;
    Counts hc;
    int herr = 0;
    if (cudaMemcpyAsync(&hc, t->d_counts, sizeof(Counts), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaMemcpyAsync(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (herr) return MGBVH_ERR_CAPACITY;  // traversal stack would have overflowed
    if (out_counts) {
        out_counts[0] = hc.nodes;
        out_counts[1] = hc.boxes;
        out_counts[2] = hc.tris;
    }
    if (out_seconds) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t->ev0, t->ev1);
        *out_seconds = ms * 1e-3;
    }
    return MGBVH_OK;
}

int mgbvh_trace_closest_dev(mgbvh_tracer* t, const float* d_rays, uint32_t n_rays, float* d_hit_t,
                            uint32_t* d_hit_prim, uint64_t* out_counts, double* out_seconds,
                            void* stream) {
    if (!t || !t->nodes || (n_rays && (!d_rays || !d_hit_t || !d_hit_prim))) return MGBVH_ERR_INVALID_ARG;
    if (n_rays == 0) return MGBVH_OK;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(t->d_counts, 0, sizeof(Counts), sm) != cudaSuccess ||
        cudaMemsetAsync(t->d_err, 0, sizeof(int), sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (int rc = ensure_order_buffers(t, n_rays)) return rc;
    cudaEventRecord(t->ev0, sm);
    const uint32_t grid = (n_rays + 127) / 128;
    const float4* nodes = reinterpret_cast<const float4*>(t->nodes);
    const float4* rays = reinterpret_cast<const float4*>(d_rays);
    const uint32_t* order = ray_order(t, rays, n_rays, sm, MGBVH_RAY_SORT_BINARY);
    Counts* cnt = out_counts ? t->d_counts : nullptr;
    if (MGBVH_TRACE_PERSISTENT) {
        cudaMemsetAsync(t->d_next, 0, 4, sm);
        const int pgrid = (int)std::min<uint32_t>(grid, (uint32_t)t->trace_blocks);
        if (t->lens)
            trace_persistent_kernel<true><<<pgrid, 128, 0, sm>>>(nodes, t->lens, t->tris, rays, n_rays, d_hit_t,
                                                                 d_hit_prim, cnt, t->d_err, order, t->d_next);
        else
            trace_persistent_kernel<false><<<pgrid, 128, 0, sm>>>(nodes, nullptr, t->tris, rays, n_rays, d_hit_t,
                                                                  d_hit_prim, cnt, t->d_err, order, t->d_next);
    } else if (t->lens) {
        trace_kernel<true><<<grid, 128, 0, sm>>>(nodes, t->lens, t->tris, rays, n_rays, d_hit_t, d_hit_prim, cnt,
                                                 t->d_err, order);
    } else {
        trace_kernel<false><<<grid, 128, 0, sm>>>(nodes, nullptr, t->tris, rays, n_rays, d_hit_t, d_hit_prim, cnt,
                                                  t->d_err, order);
    }
    cudaEventRecord(t->ev1, sm);
    if (cudaGetLastError() != cudaSuccess) return MGBVH_ERR_CUDA;
    Counts hc;
    int herr = 0;
    if (cudaMemcpyAsync(&hc, t->d_counts, sizeof(Counts), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaMemcpyAsync(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (herr) return MGBVH_ERR_CAPACITY;  // traversal stack would have overflowed
    if (out_counts) {
        out_counts[0] = hc.nodes;
        out_counts[1] = hc.boxes;
        out_counts[2] = hc.tris;
    }
    if (out_seconds) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t->ev0, t->ev1);
        *out_seconds = ms * 1e-3;
    }
    return MGBVH_OK;
}

int mgbvh_trace_bruteforce_dev(mgbvh_tracer* t, const float* d_rays, uint32_t n_rays, float* d_hit_t,
                               uint32_t* d_hit_prim, void* stream) {
    if (!t || !t->tris || (n_rays && (!d_rays || !d_hit_t || !d_hit_prim))) return MGBVH_ERR_INVALID_ARG;
    if (n_rays == 0) return MGBVH_OK;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    brute_kernel<<<(n_rays + 255) / 256, 256, 0, sm>>>(t->tris, t->n_tris,
                                                        reinterpret_cast<const float4*>(d_rays), n_rays,
                                                        d_hit_t, d_hit_prim);
    if (cudaGetLastError() != cudaSuccess) return MGBVH_ERR_CUDA;
    return trace_check(cudaStreamSynchronize(sm));
}

int mgbvh_tracer_set_scene_dev(mgbvh_tracer* t, const mgbvh_node* d_tlas_nodes, uint32_t tlas_node_count,
                               const uint32_t* d_tlas_lens, const mgbvh_scene_instance* d_instances,
                               uint32_t instance_count, const mgbvh_scene_mesh* d_meshes, uint32_t mesh_count,
                               const mgbvh_node* d_blas_nodes, uint32_t blas_node_count,
                               const uint32_t* d_blas_lens, const float* d_vertices, uint32_t vertex_stride_bytes,
                               uint32_t vertex_count, const uint32_t* d_triangles, uint32_t triangle_count,
                               void* stream) {
    static_assert(sizeof(mgbvh_scene_mesh) == sizeof(SceneMesh), "mesh record layout");
    static_assert(sizeof(mgbvh_scene_instance) == sizeof(SceneInst), "instance record layout");
    if (!t || !d_tlas_nodes || tlas_node_count == 0 || !d_instances || instance_count == 0 || !d_meshes ||
        mesh_count == 0 || mesh_count > 65535 || !d_blas_nodes || blas_node_count == 0 || !d_vertices ||
        !d_triangles || triangle_count == 0 || vertex_stride_bytes < 12 || vertex_stride_bytes % 4)
        return MGBVH_ERR_INVALID_ARG;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    // the mesh table: checked on the host, copied into the tracer
    std::vector<mgbvh_scene_mesh> hm(mesh_count);
    if (cudaMemcpyAsync(hm.data(), d_meshes, sizeof(mgbvh_scene_mesh) * mesh_count, cudaMemcpyDeviceToHost, sm) !=
            cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    uint32_t max_count = 0;
    for (const mgbvh_scene_mesh& m : hm) {
        if (m.triangle_count == 0) continue;  // an empty mesh has no BLAS; its instances hit nothing
        if ((uint64_t)m.triangle_offset + m.triangle_count > triangle_count || m.blas_root >= blas_node_count)
            return MGBVH_ERR_INVALID_ARG;
        max_count = std::max(max_count, m.triangle_count);
    }
    const size_t need = sizeof(TriRec) * (size_t)triangle_count;
    if (t->tris_cap < need) {
        if (t->tris) cudaFree(t->tris);
        t->tris = nullptr;
        t->tris_cap = 0;
        if (cudaMalloc(&t->tris, need) != cudaSuccess) return MGBVH_ERR_CUDA;
        t->tris_cap = need;
    }
    if (t->meshes_cap < mesh_count) {
        if (t->meshes) cudaFree(t->meshes);
        t->meshes = nullptr;
        t->meshes_cap = 0;
        if (cudaMalloc(&t->meshes, sizeof(SceneMesh) * mesh_count) != cudaSuccess) return MGBVH_ERR_CUDA;
        t->meshes_cap = mesh_count;
    }
    if (cudaMemcpyAsync(t->meshes, hm.data(), sizeof(SceneMesh) * mesh_count, cudaMemcpyHostToDevice, sm) !=
            cudaSuccess ||
        cudaMemsetAsync(t->d_err, 0, sizeof(int), sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    const dim3 grid(std::max(1u, std::min((max_count + 255) / 256, 64u)), mesh_count);
    gather_scene_kernel<<<grid, 256, 0, sm>>>(d_vertices, vertex_stride_bytes / 4, vertex_count, d_triangles,
                                              triangle_count, t->meshes, t->tris, t->d_err);
    int herr = 0;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (herr) return MGBVH_ERR_INVALID_ARG;
    t->scene = true;
    t->tlas = d_tlas_nodes;
    t->tlas_lens = d_tlas_lens;
    t->inst = reinterpret_cast<const SceneInst*>(d_instances);
    t->n_inst = instance_count;
    t->n_meshes = mesh_count;
    t->blas = d_blas_nodes;
    t->blas_lens = d_blas_lens;
    t->n_tris = triangle_count;
    // the one-level traversal and the wide tree no longer apply
    t->nodes = nullptr;
    t->lens = nullptr;
    t->node_count = 0;
    t->wide_count = 0;
    return MGBVH_OK;
}

int mgbvh_trace_scene_dev(mgbvh_tracer* t, const float* d_rays, uint32_t n_rays, float* d_hit_t,
                          uint32_t* d_hit_instance, uint32_t* d_hit_triangle, uint64_t* out_counts,
                          double* out_seconds, void* stream) {
    if (!t || !t->scene || (n_rays && (!d_rays || !d_hit_t || !d_hit_instance || !d_hit_triangle)))
        return MGBVH_ERR_INVALID_ARG;
    if (n_rays == 0) return MGBVH_OK;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(t->d_counts, 0, sizeof(Counts), sm) != cudaSuccess ||
        cudaMemsetAsync(t->d_err, 0, sizeof(int), sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (int rc = ensure_order_buffers(t, n_rays)) return rc;
    cudaEventRecord(t->ev0, sm);
    const float4* rays = reinterpret_cast<const float4*>(d_rays);
    const uint32_t* order = ray_order(t, rays, n_rays, sm, MGBVH_RAY_SORT_BINARY, t->tlas);
    Counts* cnt = out_counts ? t->d_counts : nullptr;
    const uint32_t grid = (n_rays + 127) / 128;
    const float4* tl = reinterpret_cast<const float4*>(t->tlas);
    const float4* bl = reinterpret_cast<const float4*>(t->blas);
    auto launch = [&](auto kern) {
        kern<<<grid, 128, 0, sm>>>(tl, t->tlas_lens, t->inst, t->n_inst, t->meshes, t->n_meshes, bl, t->blas_lens,
                                   t->tris, rays, n_rays, d_hit_t, d_hit_instance, d_hit_triangle, cnt, t->d_err,
                                   order);
    };
    if (t->tlas_lens && t->blas_lens)
        launch(trace_scene_kernel<true, true>);
    else if (t->tlas_lens)
        launch(trace_scene_kernel<true, false>);
    else if (t->blas_lens)
        launch(trace_scene_kernel<false, true>);
    else
        launch(trace_scene_kernel<false, false>);
    cudaEventRecord(t->ev1, sm);
    if (cudaGetLastError() != cudaSuccess) return MGBVH_ERR_CUDA;
    Counts hc;
    int herr = 0;
    if (cudaMemcpyAsync(&hc, t->d_counts, sizeof(Counts), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaMemcpyAsync(&herr, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, sm) != cudaSuccess ||
        cudaStreamSynchronize(sm) != cudaSuccess)
        return MGBVH_ERR_CUDA;
    if (herr == 1) return MGBVH_ERR_CAPACITY;  // traversal stack would have overflowed
    if (herr) return MGBVH_ERR_INVALID_ARG;    // a TLAS leaf names an instance or mesh past the tables
    if (out_counts) {
        out_counts[0] = hc.nodes;
        out_counts[1] = hc.boxes;
        out_counts[2] = hc.tris;
    }
    if (out_seconds) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t->ev0, t->ev1);
        *out_seconds = ms * 1e-3;
    }
    return MGBVH_OK;
}

int mgbvh_trace_scene_bruteforce_dev(mgbvh_tracer* t, const float* d_rays, uint32_t n_rays, float* d_hit_t,
                                     uint32_t* d_hit_instance, uint32_t* d_hit_triangle, int cull_by_mesh_bounds,
                                     void* stream) {
    if (!t || !t->scene || (n_rays && (!d_rays || !d_hit_t || !d_hit_instance || !d_hit_triangle)))
        return MGBVH_ERR_INVALID_ARG;
    if (n_rays == 0) return MGBVH_OK;
    if (cudaSetDevice(t->device) != cudaSuccess) return MGBVH_ERR_CUDA;
    const cudaStream_t sm = reinterpret_cast<cudaStream_t>(stream);
    brute_scene_kernel<<<std::min<uint32_t>(n_rays, 148u * 8u), kBruteThreads, 0, sm>>>(
        t->inst, t->n_inst, t->meshes, t->n_meshes, reinterpret_cast<const float4*>(t->blas), t->tris,
        reinterpret_cast<const float4*>(d_rays), n_rays, d_hit_t, d_hit_instance, d_hit_triangle,
        cull_by_mesh_bounds);
    if (cudaGetLastError() != cudaSuccess) return MGBVH_ERR_CUDA;
    return trace_check(cudaStreamSynchronize(sm));
}

}  // extern "C"
