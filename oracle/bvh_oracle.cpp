// bvh_oracle.cpp — CPU restatement of marigold's SAH BVH builder.
//
// TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA builder is
// compared against, and the timed CPU baseline. The product library never
// links, loads or calls it.
//
// PARITY UNPINNED: the reference crate (Rust nightly) cannot be compiled
// where this project is built, and the reference ships no tests, golden
// vectors or fixtures for the builder. This file restates the reference
// algorithm statement by statement; its pins are hand-worked known-answer
// trees and the reference's own release-mode invariants.
//
// Followed line by line (paths relative to the marigold repository):
//   BoundingVolume ops ............ bvh/src/lib.rs:61-111
//   DEPTH_COST / OBJECT_COST ...... bvh/src/lib.rs:217-218, leaf_cost :251-253
//   root / root_with_bounds ....... bvh/src/lib.rs:220-243
//   evaluate_binned_split ......... bvh/src/lib.rs:255-290
//   evaluate_threshold_split ...... bvh/src/lib.rs:292-329
//   binned_sweep .................. bvh/src/lib.rs:331-389
//   adaptive_sweep ................ bvh/src/lib.rs:392-442
//   median_split .................. bvh/src/lib.rs:444-491 (all three axes
//                                   reorder the same list, :528-530)
//   select_split .................. bvh/src/lib.rs:493-534
//   split ......................... bvh/src/lib.rs:537-665
//   new + stats ................... bvh/src/lib.rs:698-835
//   MeshTriangle AABB ............. mesh_interface/src/lib.rs:19-30
//
// Two list-order modes:
//   stable (parity mode): every partition keeps relative order. The reference
//     uses unstable partitions (Iterator::partition_in_place and
//     slice::select_nth_unstable_by); those fix the same SETS, so the tree is
//     the same except where list order decides: exact-cost ties between
//     different splits among the len < 8 centroid thresholds, and the object
//     order inside leaves holding more than one object. The GPU builder
//     implements exactly this mode.
//   faithful (baseline timing mode): AABBs recomputed through the index
//     gather on every access, two-ended partition_in_place, nth_element for
//     index/median splits, and the assertion passes — the algorithmic form of
//     the Rust code, for timing.
//
// Build flags: -O3 -ffp-contract=off, no -ffast-math: every f32 operation is
// one IEEE single-precision operation in the reference's order.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#include "../include/mgbvh.h"

namespace {

constexpr float kDepthCost = 1.0f;   // bvh/src/lib.rs:217
constexpr float kObjectCost = 8.0f;  // bvh/src/lib.rs:218
constexpr float kInf = std::numeric_limits<float>::infinity();

// Tie events of the last build on this thread: equal-cost len<8 centroid
// thresholds that split different object sets (the only place where list
// order, not the object set, picks the split).
thread_local uint32_t g_tie_events = 0;
// Nodes of the last build on this thread whose split was one of several
// equal-cost splits over different object sets on the winning axis, chosen by
// list order: the nodes where the reference's unstable partitions
// (partition_in_place, select_nth_unstable_by) could make its tree differ.
thread_local uint32_t g_order_dependent = 0;

// glam's SSE2 Vec3A::min/max are _mm_min_ps/_mm_max_ps: a < b ? a : b.
inline float vmin(float a, float b) { return a < b ? a : b; }
inline float vmax(float a, float b) { return a > b ? a : b; }

struct BV {
    float mn[3];
    float mx[3];
};

inline BV bv_empty() { return BV{{kInf, kInf, kInf}, {-kInf, -kInf, -kInf}}; }

inline void bv_grow(BV& b, const BV& o) {  // :98-101
    for (int a = 0; a < 3; ++a) {
        b.mn[a] = vmin(b.mn[a], o.mn[a]);
        b.mx[a] = vmax(b.mx[a], o.mx[a]);
    }
}

inline float bv_center(const BV& b, int a) { return (b.mn[a] + b.mx[a]) * 0.5f; }  // :71-73

inline bool bv_is_empty(const BV& b) {  // :103-106
    return b.mx[0] < b.mn[0] || b.mx[1] < b.mn[1] || b.mx[2] < b.mn[2];
}

inline float bv_surface_area(const BV& b) {  // :79-91
    float w = b.mx[0] - b.mn[0];
    float h = b.mx[1] - b.mn[1];
    float d = b.mx[2] - b.mn[2];
    if (!bv_is_empty(b)) {
        float s = w * h;
        s = s + w * d;
        s = s + h * d;
        return 2.0f * s;
    }
    return 0.0f;
}

inline bool bv_contains(const BV& b, const float p[3]) {  // :108-110
    return !bv_is_empty(b) && p[0] >= b.mn[0] && p[1] >= b.mn[1] && p[2] >= b.mn[2] &&
           p[0] <= b.mx[0] && p[1] <= b.mx[1] && p[2] <= b.mx[2];
}

// f32::total_cmp as an unsigned key: same order, NaNs at the ends by sign.
inline uint32_t total_key(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// cost formula of :278-288 / :317-327 / :470-482, evaluated in that order
inline float split_cost(float sa_lt, float sa_gt, float sa_parent, uint32_t cnt_lt,
                        uint32_t cnt_gt) {
    float lt_cost = sa_lt / sa_parent * kObjectCost * static_cast<float>(cnt_lt);
    float gt_cost = sa_gt / sa_parent * kObjectCost * static_cast<float>(cnt_gt);
    return kDepthCost + lt_cost + gt_cost;
}

enum Kind : uint8_t { kThreshold = 0, kIndex = 1, kExact = 2 };

struct Split {
    BV lt, gt;
    uint32_t cnt_lt, cnt_gt;
    float cost;
    Kind kind;
    int axis;
    float threshold;
    uint32_t index;
    // len < 8 adaptive split whose axis holds another threshold of the same
    // cost over a different object set: list order picked this one
    bool order_dep = false;
};

struct Node {
    BV bounds;
    uint32_t start, len, child;
};

// Object accessors: the AsBoundingVolumeIndices impls.
struct IndexedAcc {  // MeshTriangle over MeshVertex, mesh_interface/src/lib.rs:19-30
    const float* verts;
    uint32_t stride;  // in floats
    const uint32_t* tris;
    BV operator()(uint32_t id) const {
        const float* p0 = verts + static_cast<size_t>(tris[3 * (size_t)id + 0]) * stride;
        const float* p1 = verts + static_cast<size_t>(tris[3 * (size_t)id + 1]) * stride;
        const float* p2 = verts + static_cast<size_t>(tris[3 * (size_t)id + 2]) * stride;
        BV b;
        for (int a = 0; a < 3; ++a) {
            // +0.0 turns a -0.0 input into +0.0 (the builder's one input rule)
            const float x0 = p0[a] + 0.0f, x1 = p1[a] + 0.0f, x2 = p2[a] + 0.0f;
            b.mn[a] = vmin(vmin(x0, x1), x2);
            b.mx[a] = vmax(vmax(x0, x1), x2);
        }
        return b;
    }
};

struct AabbAcc {  // AsBoundingVolume objects given by their AABB
    const float* aabbs;
    BV operator()(uint32_t id) const {
        const float* p = aabbs + 6 * (size_t)id;
        return BV{{p[0] + 0.0f, p[1] + 0.0f, p[2] + 0.0f}, {p[3] + 0.0f, p[4] + 0.0f, p[5] + 0.0f}};
    }
};

struct CachedAcc {  // precomputed AABBs (parity mode; identical values)
    const BV* b;
    BV operator()(uint32_t id) const { return b[id]; }
};

struct Knobs {
    uint32_t bins, adaptive_max_n, adaptive_steps;
    uint32_t full_sweep;  // every node: every centroid a threshold on every axis
    // the learned form with fixed proposals (learn_max_n 0: off): at every
    // binned node of 33..learn_max_n objects, 16 thresholds inside each of
    // the two (axis * 16 + bucket) proposals replace the binned split when
    // strictly cheaper
    uint32_t learn_max_n;
    uint32_t prop[2];
};

template <class Acc, bool kFaithful>
struct Builder {
    const Acc& acc;
    uint32_t MIN, MAX, max_depth;
    Knobs k;
    std::vector<uint32_t> list;
    std::vector<Node> nodes;
    uint32_t height = 0;
    // node samples for the learned split proposer (features + full-sweep label)
    std::vector<float>* samples = nullptr;
    uint32_t sample_min_n = 33;
    uint32_t median_splits = 0, tie_events = 0, depth_capped = 0, learned_splits = 0, order_dependent = 0;
    int error = 0;

    Builder(const Acc& a, uint32_t mn, uint32_t mx, uint32_t md, Knobs kn)
        : acc(a), MIN(mn), MAX(mx), max_depth(md), k(kn) {}

    float center(uint32_t id, int a) const { return bv_center(acc(id), a); }

    // ---- evaluate_threshold_split, :292-329
    Split eval_threshold(const BV& parent, uint32_t s, uint32_t n, int axis, float thr) const {
        Split sp{};
        sp.lt = bv_empty();
        sp.gt = bv_empty();
        sp.cnt_lt = sp.cnt_gt = 0;
        for (uint32_t i = s; i < s + n; ++i) {
            BV b = acc(list[i]);
            if (bv_center(b, axis) < thr) {
                bv_grow(sp.lt, b);
                sp.cnt_lt++;
            } else {
                bv_grow(sp.gt, b);
                sp.cnt_gt++;
            }
        }
        sp.cost = split_cost(bv_surface_area(sp.lt), bv_surface_area(sp.gt),
                             bv_surface_area(parent), sp.cnt_lt, sp.cnt_gt);
        sp.kind = kThreshold;
        sp.axis = axis;
        sp.threshold = thr;
        return sp;
    }

    // min_by(total_cmp): replace only when strictly smaller (first minimum wins)
    static bool better(const Split& cand, const Split& best) {
        return total_key(cand.cost) < total_key(best.cost);
    }

    // ---- binned_sweep, :331-389
    bool binned_sweep(const BV& parent, const BV& cb, uint32_t s, uint32_t n, int axis,
                      Split& out) const {
        float ext = cb.mx[axis] - cb.mn[axis];
        if (ext == 0.0f) return false;  // :339
        uint32_t bin_count = k.bins ? k.bins : std::clamp<uint32_t>(n, 16, 32);  // :343
        struct Bin {
            uint32_t count;
            BV b;
        };
        std::vector<Bin> bins(bin_count, Bin{0, bv_empty()});
        for (uint32_t i = s; i < s + n; ++i) {  // :354-368
            BV ob = acc(list[i]);
            float c = bv_center(ob, axis);
            float pct = (c - cb.mn[axis]) / (cb.mx[axis] - cb.mn[axis]);
            float f = std::floor(pct * static_cast<float>(bin_count));
            // `as usize` saturates: NaN and negatives become 0
            size_t bi = (f != f || f <= 0.0f) ? 0 : (f >= 4294967296.0f ? SIZE_MAX : (size_t)f);
            bi = std::min<size_t>(bi, bin_count - 1);
            bins[bi].count++;
            bv_grow(bins[bi].b, ob);
        }
        bool found = false;
        float sa_p = bv_surface_area(parent);
        for (uint32_t i = 1; i < bin_count; ++i) {  // :373-388
            // evaluate_binned_split, :255-290 — re-merged per candidate
            Split sp{};
            sp.lt = bv_empty();
            sp.gt = bv_empty();
            sp.cnt_lt = sp.cnt_gt = 0;
            for (uint32_t j = 0; j < i; ++j) {
                sp.cnt_lt += bins[j].count;
                bv_grow(sp.lt, bins[j].b);
            }
            for (uint32_t j = i; j < bin_count; ++j) {
                sp.cnt_gt += bins[j].count;
                bv_grow(sp.gt, bins[j].b);
            }
            sp.cost = split_cost(bv_surface_area(sp.lt), bv_surface_area(sp.gt), sa_p, sp.cnt_lt,
                                 sp.cnt_gt);
            if (sp.cnt_lt < MIN || sp.cnt_gt < MIN) continue;  // :379
            sp.kind = kIndex;
            sp.axis = axis;
            sp.index = sp.cnt_lt;  // :376
            sp.threshold = 0.0f;
            if (!found || better(sp, out)) {
                out = sp;
                found = true;
            }
        }
        return found;
    }

    // ---- adaptive_sweep, :392-442
    bool adaptive_sweep(const BV& parent, const BV& cb, uint32_t s, uint32_t n, int axis,
                        Split& out) {
        const uint32_t accurate = 8;  // :399
        bool found = false;
        if (n < accurate) {
            // one threshold per object centroid, in list order (:417-427)
            for (uint32_t i = s; i < s + n; ++i) {
                float thr = center(list[i], axis);
                Split sp = eval_threshold(parent, s, n, axis, thr);
                if (sp.cnt_lt < MIN || sp.cnt_gt < MIN) continue;
                if (!found) {
                    out = sp;
                    found = true;
                } else if (better(sp, out)) {
                    out = sp;
                } else if (total_key(sp.cost) == total_key(out.cost) &&
                           sp.threshold != out.threshold) {
                    // equal cost: does a different object set lie between?
                    float lo = std::min(sp.threshold, out.threshold);
                    float hi = std::max(sp.threshold, out.threshold);
                    for (uint32_t j = s; j < s + n; ++j) {
                        float c = center(list[j], axis);
                        if (c >= lo && c < hi) {
                            tie_events++;
                            out.order_dep = true;
                            break;
                        }
                    }
                }
            }
        } else {
            uint32_t step_count =
                k.adaptive_steps ? k.adaptive_steps : std::clamp<uint32_t>(n, accurate, 32);  // :430
            float bounds_step = (cb.mx[axis] - cb.mn[axis]) / static_cast<float>(step_count);
            for (uint32_t i = 0; i < step_count; ++i) {
                float thr = cb.mn[axis] + bounds_step * (static_cast<float>(i) + 0.5f);  // :436
                Split sp = eval_threshold(parent, s, n, axis, thr);
                if (sp.cnt_lt < MIN || sp.cnt_gt < MIN) continue;
                if (!found || better(sp, out)) {
                    out = sp;
                    found = true;
                }
            }
        }
        return found;
    }

    // Stable restatement of select_nth_unstable_by(m, total_cmp on centroid):
    // the m smallest keys (ties by list position) move to the front, each side
    // keeping its relative order.
    void stable_select(uint32_t s, uint32_t n, int axis, uint32_t m) {
        std::vector<std::pair<uint64_t, uint32_t>> keyed(n);
        for (uint32_t i = 0; i < n; ++i)
            keyed[i] = {((uint64_t)total_key(center(list[s + i], axis)) << 32) | i, i};
        std::vector<uint8_t> lt(n, 0);
        if (m > 0 && m <= n) {
            std::nth_element(keyed.begin(), keyed.begin() + (m - 1), keyed.end());
            uint64_t cut = keyed[m - 1].first;
            for (uint32_t i = 0; i < n; ++i) {
                uint64_t key = ((uint64_t)total_key(center(list[s + i], axis)) << 32) | i;
                lt[i] = key <= cut;
            }
        }
        std::vector<uint32_t> tmp;
        tmp.reserve(n);
        for (uint32_t i = 0; i < n; ++i)
            if (lt[i]) tmp.push_back(list[s + i]);
        for (uint32_t i = 0; i < n; ++i)
            if (!lt[i]) tmp.push_back(list[s + i]);
        std::copy(tmp.begin(), tmp.end(), list.begin() + s);
    }

    void nth_select(uint32_t s, uint32_t n, int axis, uint32_t m) {
        if (m >= n) return;
        std::nth_element(list.begin() + s, list.begin() + s + m, list.begin() + s + n,
                         [&](uint32_t a, uint32_t b) {
                             return total_key(center(a, axis)) < total_key(center(b, axis));
                         });
    }

    // ---- median_split, :444-491
    Split median_split(const BV& parent, uint32_t s, uint32_t n, int axis) {
        uint32_t m = n / 2;
        if (kFaithful)
            nth_select(s, n, axis, m);
        else
            stable_select(s, n, axis, m);
        Split sp{};
        sp.lt = bv_empty();
        sp.gt = bv_empty();
        for (uint32_t i = s; i < s + m; ++i) bv_grow(sp.lt, acc(list[i]));
        for (uint32_t i = s + m; i < s + n; ++i) bv_grow(sp.gt, acc(list[i]));
        sp.cnt_lt = m;
        sp.cnt_gt = n - m;
        sp.cost = split_cost(bv_surface_area(sp.lt), bv_surface_area(sp.gt),
                             bv_surface_area(parent), m, n - m);
        sp.kind = kExact;
        sp.axis = axis;
        sp.index = m;
        return sp;
    }

    // Exact sweep (not in the reference; the quality yardstick of the learned
    // proposer): on each axis, every distinct centroid value is a threshold
    // (lt = centroids strictly below it), scored with the reference's cost
    // formula; first minimum over (cost, axis, threshold rank) wins.
    bool full_sweep(const BV& parent, uint32_t s, uint32_t n, Split& out) {
        const float sa_p = bv_surface_area(parent);
        std::vector<std::pair<float, uint32_t>> key(n);
        std::vector<BV> pre(n), suf(n);
        bool found = false;
        for (int axis = 0; axis < 3; ++axis) {
            for (uint32_t i = 0; i < n; ++i) key[i] = {center(list[s + i], axis), list[s + i]};
            std::stable_sort(key.begin(), key.end(),
                             [](const auto& a, const auto& b) { return total_key(a.first) < total_key(b.first); });
            BV acc = bv_empty();
            for (uint32_t i = 0; i < n; ++i) {
                bv_grow(acc, acc_box(key[i].second));
                pre[i] = acc;
            }
            acc = bv_empty();
            for (uint32_t i = n; i-- > 0;) {
                bv_grow(acc, acc_box(key[i].second));
                suf[i] = acc;
            }
            for (uint32_t i = 1; i < n; ++i) {
                if (!(key[i - 1].first < key[i].first)) continue;  // same centroid: same set
                const uint32_t nl = i, ng = n - i;
                if (nl < MIN || ng < MIN) continue;
                Split sp{};
                sp.lt = pre[i - 1];
                sp.gt = suf[i];
                sp.cnt_lt = nl;
                sp.cnt_gt = ng;
                sp.cost = split_cost(bv_surface_area(sp.lt), bv_surface_area(sp.gt), sa_p, nl, ng);
                sp.kind = kThreshold;
                sp.axis = axis;
                sp.threshold = key[i].first;
                if (!found || better(sp, out)) {
                    out = sp;
                    found = true;
                }
            }
        }
        return found;
    }

    BV acc_box(uint32_t id) const { return acc(id); }

    // One training sample per node: 24 features, then the label: the
    // full-sweep optimum's axis * 16 + position bucket (16 equal buckets over
    // the centroid extent), whether it beats the plain split's cost, the
    // object count, both costs and the node's start in the object list. Feature order (all finite):
    //   0-2  node extent / largest node extent
    //   3-5  centroid extent / largest node extent
    //   6    log2(n) / 20
    //   7-18 per axis, the fraction of centroids in 4 equal buckets of the
    //        centroid extent (floor(4 * (c - cmin) / ext), clamped)
    //   19   SA(centroid bounds) / SA(node)
    //   20   depth / 32
    //   21   middle / largest node extent, 22 smallest / largest node extent
    //   23   largest centroid extent / largest node extent
    void record_sample(const BV& parent, uint32_t s, uint32_t n, uint32_t depth) {
        float cmn[3] = {kInf, kInf, kInf}, cmx[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = s; i < s + n; ++i) {
            BV b = acc(list[i]);
            for (int a = 0; a < 3; ++a) {
                const float c = bv_center(b, a);
                cmn[a] = vmin(cmn[a], c);
                cmx[a] = vmax(cmx[a], c);
            }
        }
        float f[24] = {0};
        float ext[3], cext[3];
        for (int a = 0; a < 3; ++a) {
            ext[a] = parent.mx[a] - parent.mn[a];
            cext[a] = cmx[a] - cmn[a];
        }
        const float emax = std::max(std::max(ext[0], ext[1]), std::max(ext[2], 1e-30f));
        for (int a = 0; a < 3; ++a) {
            f[a] = ext[a] / emax;
            f[3 + a] = cext[a] / emax;
        }
        f[6] = std::log2((float)n) / 20.0f;
        for (uint32_t i = s; i < s + n; ++i) {
            BV b = acc(list[i]);
            for (int a = 0; a < 3; ++a) {
                if (!(cext[a] > 0.0f)) continue;
                const float pct = (bv_center(b, a) - cmn[a]) / cext[a];
                int q = (int)std::floor(pct * 4.0f);
                q = std::min(std::max(q, 0), 3);
                f[7 + 4 * a + q] += 1.0f;
            }
        }
        for (int j = 7; j < 19; ++j) f[j] /= (float)n;
        BV cb{{cmn[0], cmn[1], cmn[2]}, {cmx[0], cmx[1], cmx[2]}};
        const float sap = bv_surface_area(parent);
        f[19] = sap > 0.0f ? bv_surface_area(cb) / sap : 0.0f;
        f[20] = (float)depth / 32.0f;
        float e[3] = {ext[0], ext[1], ext[2]};
        std::sort(e, e + 3);
        f[21] = e[1] / emax;
        f[22] = e[0] / emax;
        f[23] = std::max(std::max(cext[0], cext[1]), cext[2]) / emax;
        Split plain, best;
        const bool okp = select_split_plain(parent, s, n, plain);
        const bool okf = full_sweep(parent, s, n, best);
        uint32_t label = 0xFFFFFFFFu, gain = 0;
        if (okf && cext[best.axis] > 0.0f) {
            const float pct = (best.threshold - cmn[best.axis]) / cext[best.axis];
            int q = (int)std::floor(pct * 16.0f);
            q = std::min(std::max(q, 0), 15);
            label = (uint32_t)best.axis * 16u + (uint32_t)q;
            gain = (!okp || total_key(best.cost) < total_key(plain.cost)) ? 1u : 0u;
        }
        for (int j = 0; j < 24; ++j) samples->push_back(f[j]);
        uint32_t lb = label;
        float w;
        std::memcpy(&w, &lb, 4);
        samples->push_back(w);
        samples->push_back((float)gain);
        samples->push_back((float)n);
        samples->push_back(okp ? plain.cost : kInf);
        samples->push_back(okf ? best.cost : kInf);
        samples->push_back((float)s);
    }

    // The learned form's split rule (not in the reference), for two given
    // proposals: lane p * 16 + k (p = proposal, k = 0..15) tries the
    // threshold cmin + ext * ((bucket * 16 + k + 1) / 256) on the proposal's
    // axis; the first minimum of (cost, axis, lane) replaces the binned split
    // when its cost is strictly below the binned cost.
    void learned_refine(const BV& parent, uint32_t s, uint32_t n, Split& sp) {
        float cmn[3] = {kInf, kInf, kInf}, cmx[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = s; i < s + n; ++i) {
            BV b = acc(list[i]);
            for (int a = 0; a < 3; ++a) {
                const float c = bv_center(b, a);
                cmn[a] = vmin(cmn[a], c);
                cmx[a] = vmax(cmx[a], c);
            }
        }
        uint64_t best = ~0ull;
        Split bsp{};
        for (uint32_t lane = 0; lane < 32; ++lane) {
            const uint32_t prop = k.prop[lane >> 4];
            const int a = (int)(prop >> 4);
            const uint32_t bucket = prop & 15u, kk = lane & 15u;
            const float ext = cmx[a] - cmn[a];
            if (!(ext > 0.0f)) continue;
            const float thr = cmn[a] + ext * ((float)(bucket * 16u + kk + 1u) / 256.0f);
            Split c = eval_threshold(parent, s, n, a, thr);
            if (c.cnt_lt < MIN || c.cnt_gt < MIN) continue;
            const uint64_t key = ((uint64_t)total_key(c.cost) << 32) | ((uint64_t)a << 8) | lane;
            if (key < best) {
                best = key;
                bsp = c;
            }
        }
        if (best != ~0ull && (uint32_t)(best >> 32) < total_key(sp.cost)) {
            sp = bsp;
            learned_splits++;
        }
    }

    // select_split without the full-sweep switch and without side effects on
    // the list (binned / adaptive only; the median is not needed for labels)
    bool select_split_plain(const BV& parent, uint32_t s, uint32_t n, Split& out) {
        float cmn[3] = {kInf, kInf, kInf}, cmx[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = s; i < s + n; ++i) {
            BV b = acc(list[i]);
            for (int a = 0; a < 3; ++a) {
                const float c = bv_center(b, a);
                cmn[a] = vmin(cmn[a], c);
                cmx[a] = vmax(cmx[a], c);
            }
        }
        BV cb{{cmn[0], cmn[1], cmn[2]}, {cmx[0], cmx[1], cmx[2]}};
        bool found = false;
        for (int axis = 0; axis < 3; ++axis) {
            Split sp;
            const bool ok = (n <= k.adaptive_max_n) ? adaptive_sweep(parent, cb, s, n, axis, sp)
                                                    : binned_sweep(parent, cb, s, n, axis, sp);
            if (ok && (!found || better(sp, out))) {
                out = sp;
                found = true;
            }
        }
        return found;
    }

    // ---- select_split, :493-534
    bool select_split(const BV& parent, uint32_t s, uint32_t n, Split& out) {
        if (k.full_sweep) {
            if (full_sweep(parent, s, n, out)) return true;
            if (n <= MAX) return false;
            bool found = false;  // coincident centroids: the forced median as below
            for (int axis = 0; axis < 3; ++axis) {
                Split sp = median_split(parent, s, n, axis);
                if (!found || better(sp, out)) {
                    out = sp;
                    found = true;
                }
            }
            median_splits++;
            return found;
        }
        float cmn[3] = {kInf, kInf, kInf}, cmx[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = s; i < s + n; ++i) {
            BV b = acc(list[i]);
            for (int a = 0; a < 3; ++a) {
                float c = bv_center(b, a);
                cmn[a] = vmin(cmn[a], c);
                cmx[a] = vmax(cmx[a], c);
            }
        }
        BV cb{{cmn[0], cmn[1], cmn[2]}, {cmx[0], cmx[1], cmx[2]}};
        bool found = false;
        for (int axis = 0; axis < 3; ++axis) {
            Split sp;
            bool ok = (n <= k.adaptive_max_n) ? adaptive_sweep(parent, cb, s, n, axis, sp)
                                              : binned_sweep(parent, cb, s, n, axis, sp);
            if (ok && (!found || better(sp, out))) {
                out = sp;
                found = true;
            }
        }
        if (!found && n > MAX) {  // :527-531
            for (int axis = 0; axis < 3; ++axis) {
                Split sp = median_split(parent, s, n, axis);
                if (!found || better(sp, out)) {
                    out = sp;
                    found = true;
                }
            }
            median_splits++;
        }
        return found;
    }

    // Rust's Iterator::partition_in_place: repeatedly swap the first element
    // failing the predicate with the last one passing it.
    template <class P>
    uint32_t partition_two_ended(uint32_t s, uint32_t n, P pred) {
        uint32_t lo = s, hi = s + n;
        uint32_t true_count = 0;
        while (true) {
            while (lo < hi && pred(list[lo])) {
                ++lo;
                ++true_count;
            }
            if (lo == hi) break;
            // list[lo] is false; find the last true
            uint32_t r = hi;
            bool got = false;
            while (r > lo + 1) {
                --r;
                if (pred(list[r])) {
                    got = true;
                    break;
                }
            }
            if (!got) break;
            std::swap(list[lo], list[r]);
            ++true_count;
            ++lo;
            hi = r;
        }
        return true_count;
    }

    template <class P>
    uint32_t partition_stable(uint32_t s, uint32_t n, P pred) {
        std::vector<uint32_t> a, b;
        a.reserve(n);
        b.reserve(n);
        for (uint32_t i = s; i < s + n; ++i) (pred(list[i]) ? a : b).push_back(list[i]);
        std::copy(a.begin(), a.end(), list.begin() + s);
        std::copy(b.begin(), b.end(), list.begin() + s + a.size());
        return (uint32_t)a.size();
    }

    // ---- split, :537-665, as an explicit stack in the same visiting order
    void build(Node root) {
        nodes.push_back(root);
        struct Task {
            uint32_t idx, depth;
        };
        std::vector<Task> stack;
        stack.push_back({0, 0});
        while (!stack.empty() && !error) {
            Task t = stack.back();
            stack.pop_back();
            Node self = nodes[t.idx];
            uint32_t depth = t.depth;
            if (self.len <= 1) continue;  // :548
            if (depth == max_depth || (self.len <= MAX && self.len < MIN * 2)) {  // :556
                if (self.len > 1 && depth == max_depth) depth_capped++;
                continue;
            }
            uint32_t s = self.start, n = self.len;
            if (samples && n >= sample_min_n) record_sample(self.bounds, s, n, depth);
            Split sp;
            if (!select_split(self.bounds, s, n, sp)) continue;  // :576-579
            // :583 (leaf_cost, :251-253); a NaN cost compares false and splits
            if (self.len <= MAX && sp.cost >= kObjectCost * static_cast<float>(self.len)) continue;
            if (sp.order_dep) order_dependent++;
            if (k.learn_max_n && !k.full_sweep && n > 32 && n <= k.learn_max_n && sp.kind == kIndex &&
                (k.bins ? k.bins : std::clamp<uint32_t>(n, 16, 32)) == 32)
                learned_refine(self.bounds, s, n, sp);
            uint32_t split_index;
            if (sp.kind == kThreshold) {  // :598-600
                int ax = sp.axis;
                float thr = sp.threshold;
                auto pred = [&](uint32_t id) { return center(id, ax) < thr; };
                split_index = kFaithful ? partition_two_ended(s, n, pred)
                                        : partition_stable(s, n, pred);
            } else if (sp.kind == kIndex) {  // :601-608
                if (kFaithful)
                    nth_select(s, n, sp.axis, sp.index);
                else
                    stable_select(s, n, sp.axis, sp.index);
                split_index = sp.index;
            } else {
                split_index = sp.index;  // :609
            }
            // release-mode assertions, :615-646
            uint32_t n_lt = split_index, n_gt = n - split_index;
            if (n_lt == 0 || n_gt == 0 || sp.cnt_lt != n_lt || sp.cnt_gt != n_gt) {
                error = MGBVH_ERR_ASSERT;
                break;
            }
            for (uint32_t i = s; i < s + n; ++i) {
                BV b = acc(list[i]);
                float c[3] = {bv_center(b, 0), bv_center(b, 1), bv_center(b, 2)};
                if (!bv_contains(i < s + n_lt ? sp.lt : sp.gt, c)) {
                    error = MGBVH_ERR_ASSERT;
                    break;
                }
            }
            if (error) break;
            Node gt{sp.gt, s + sp.cnt_lt, sp.cnt_gt, 0};  // :648
            Node lt{sp.lt, s, sp.cnt_lt, 0};
            uint32_t child = (uint32_t)nodes.size();  // :651
            nodes[t.idx].child = child;
            nodes.push_back(gt);
            nodes.push_back(lt);
            height = std::max(height, depth);  // :656
            stack.push_back({child + 1, depth + 1});  // lt after gt (:659-660)
            stack.push_back({child, depth + 1});
        }
    }
};

template <class Acc, bool kFaithful>
int run_build(const Acc& acc, uint32_t n, const float* root_bounds, uint32_t MIN, uint32_t MAX,
              uint32_t max_depth, Knobs kn, uint32_t* out_nodes, uint32_t node_capacity,
              uint32_t* out_lens, uint32_t* out_perm, uint32_t* out_count, mgbvh_stats* st) {
    Builder<Acc, kFaithful> b(acc, MIN, MAX, max_depth, kn);
    bool feasible = (MIN == MAX) ? (n % MIN == 0) : (MAX >= 2 * MIN - 1);  // :710-714
    auto t0 = std::chrono::steady_clock::now();
    b.list.resize(n);
    std::iota(b.list.begin(), b.list.end(), 0u);
    Node root{};
    if (root_bounds) {  // :731-735
        root.bounds = BV{{root_bounds[0], root_bounds[1], root_bounds[2]},
                         {root_bounds[3], root_bounds[4], root_bounds[5]}};
    } else {
        root.bounds = bv_empty();
        for (uint32_t i = 0; i < n; ++i) bv_grow(root.bounds, acc(i));
    }
    root.start = 0;
    root.len = n;
    root.child = 0;
    size_t cap = 2 * (((size_t)n + MAX - 1) / MAX) - 1;  // :743-748
    b.nodes.reserve(cap);
    b.build(root);
    auto t1 = std::chrono::steady_clock::now();
    if (b.error) return b.error;
    if (b.nodes.size() > node_capacity) return MGBVH_ERR_CAPACITY;
    for (size_t i = 0; i < b.nodes.size(); ++i) {
        const Node& nd = b.nodes[i];
        uint32_t* w = out_nodes + 8 * i;
        std::memcpy(w + 0, nd.bounds.mn, 12);
        w[3] = nd.start;
        std::memcpy(w + 4, nd.bounds.mx, 12);
        w[7] = nd.child;
        if (out_lens) out_lens[i] = nd.len;
    }
    if (out_perm) std::memcpy(out_perm, b.list.data(), 4 * (size_t)n);
    *out_count = (uint32_t)b.nodes.size();
    if (st) {  // :767-788
        std::memset(st, 0, sizeof(*st));
        st->construction_time = std::chrono::duration<double>(t1 - t0).count();
        std::vector<uint32_t> leaf;
        for (size_t i = 1; i < b.nodes.size(); ++i)
            if (b.nodes[i].child == 0) leaf.push_back(b.nodes[i].len);
        st->leaf_node_count = (uint32_t)leaf.size();
        st->min_leaf_object_count = leaf.empty() ? root.len : *std::min_element(leaf.begin(), leaf.end());
        st->max_leaf_object_count = leaf.empty() ? root.len : *std::max_element(leaf.begin(), leaf.end());
        uint32_t sum = 0;
        for (uint32_t l : leaf) sum += l;
        double avg = (double)sum / (double)leaf.size();
        double var = 0.0;
        for (uint32_t l : leaf) var += ((double)l - avg) * ((double)l - avg);
        st->avg_leaf_object_count = avg;
        st->stddev_leaf_object_count = std::sqrt(var / (double)leaf.size());
        st->node_count = (uint32_t)b.nodes.size();
        st->total_object_count = n;
        st->height = b.height;
        st->max_depth = max_depth;
        st->median_splits = b.median_splits;
        st->learned_splits = b.learned_splits;
        st->depth_capped_leaves = b.depth_capped;
        st->feasible = feasible;
    }
    g_tie_events = b.tie_events;
    g_order_dependent = b.order_dependent;
    return feasible ? MGBVH_OK : MGBVH_WARN_INFEASIBLE;
}

// Moller-Trumbore as marigold/assets/shaders/slang/lib/scene.slang:19-89
// evaluates it (|det| < 1e-6 and t < 1e-6 reject), every product and sum as
// written; returns t or -1 (miss).
float moller_trumbore(float ox, float oy, float oz, float dx, float dy, float dz, const float* a, const float* b,
                      const float* c) {
    auto dot3 = [](float ax, float ay, float az, float bx, float by, float bz) {
        float d = ax * bx;
        d = d + ay * by;
        d = d + az * bz;
        return d;
    };
    const float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
    const float e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
    const float hx = dy * e2z - dz * e2y, hy = dz * e2x - dx * e2z, hz = dx * e2y - dy * e2x;
    const float det = dot3(hx, hy, hz, e1x, e1y, e1z);
    if (std::fabs(det) < 1e-6f) return -1.0f;
    const float f = 1.0f / det;
    const float sx = ox - a[0], sy = oy - a[1], sz = oz - a[2];
    const float u = f * dot3(sx, sy, sz, hx, hy, hz);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const float qx = sy * e1z - sz * e1y, qy = sz * e1x - sx * e1z, qz = sx * e1y - sy * e1x;
    const float v = f * dot3(dx, dy, dz, qx, qy, qz);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = f * dot3(e2x, e2y, e2z, qx, qy, qz);
    if (t < 1e-6f) return -1.0f;
    return t;
}

}  // namespace

extern "C" {

typedef struct oracle_knobs {
    uint32_t bins, adaptive_max_n, adaptive_steps, faithful, full_sweep;
    uint32_t learn_max_n, prop0, prop1;  // the learned form with fixed proposals (0: off)
} oracle_knobs;

// Builds with the oracle. Exactly one of (verts, tris) or aabbs is given.
// out_nodes: node_capacity * 8 u32 words, the mgbvh_node layout.
int oracle_build(const float* verts, uint32_t vertex_stride_bytes, const uint32_t* tris,
                 const float* aabbs, uint32_t n, const float* root_bounds, uint32_t min_leaf,
                 uint32_t max_leaf, uint32_t max_depth, const oracle_knobs* kn,
                 uint32_t* out_nodes, uint32_t node_capacity, uint32_t* out_lens,
                 uint32_t* out_perm, uint32_t* out_count, mgbvh_stats* st) {
    if (!out_nodes || !out_count || min_leaf < 1 || max_leaf < 1) return MGBVH_ERR_INVALID_ARG;
    if ((verts == nullptr) == (aabbs == nullptr)) return MGBVH_ERR_INVALID_ARG;
    if (verts && (!tris || vertex_stride_bytes % 4 || vertex_stride_bytes < 12))
        return MGBVH_ERR_INVALID_ARG;
    *out_count = 0;
    if (n == 0) {
        if (st) std::memset(st, 0, sizeof(*st));
        return MGBVH_WARN_EMPTY;
    }
    Knobs k{kn ? kn->bins : 0, kn ? kn->adaptive_max_n : 32, kn ? kn->adaptive_steps : 0,
            kn ? kn->full_sweep : 0, kn ? kn->learn_max_n : 0,
            {kn ? kn->prop0 % 48u : 0, kn ? kn->prop1 % 48u : 0}};
    bool faithful = kn && kn->faithful;
    if (verts) {
        IndexedAcc acc{verts, vertex_stride_bytes / 4, tris};
        if (faithful)
            return run_build<IndexedAcc, true>(acc, n, root_bounds, min_leaf, max_leaf, max_depth,
                                               k, out_nodes, node_capacity, out_lens, out_perm,
                                               out_count, st);
        std::vector<BV> cache(n);
        for (uint32_t i = 0; i < n; ++i) cache[i] = acc(i);
        CachedAcc c{cache.data()};
        return run_build<CachedAcc, false>(c, n, root_bounds, min_leaf, max_leaf, max_depth, k,
                                           out_nodes, node_capacity, out_lens, out_perm,
                                           out_count, st);
    }
    AabbAcc acc{aabbs};
    if (faithful)
        return run_build<AabbAcc, true>(acc, n, root_bounds, min_leaf, max_leaf, max_depth, k,
                                        out_nodes, node_capacity, out_lens, out_perm, out_count,
                                        st);
    return run_build<AabbAcc, false>(acc, n, root_bounds, min_leaf, max_leaf, max_depth, k,
                                     out_nodes, node_capacity, out_lens, out_perm, out_count, st);
}

uint32_t oracle_last_tie_events(void) { return g_tie_events; }
uint32_t oracle_last_order_dependent(void) { return g_order_dependent; }

// Node samples of a plain (reference-profile) build over triangles: 30 floats
// per node with at least min_n objects (24 features, label as u32 bits, gain
// flag, n, plain cost, full-sweep cost, start). Returns the number of samples
// written (at most capacity).
uint32_t oracle_sample_nodes(const float* verts, uint32_t vertex_stride_bytes, const uint32_t* tris,
                             uint32_t n, uint32_t min_n, float* out, uint32_t capacity) {
    IndexedAcc acc0{verts, vertex_stride_bytes / 4, tris};
    std::vector<BV> cache(n);
    for (uint32_t i = 0; i < n; ++i) cache[i] = acc0(i);
    CachedAcc acc{cache.data()};
    Builder<CachedAcc, false> b(acc, 1, 1, 32, Knobs{0, 32, 0, 0, 0, {0, 0}});
    std::vector<float> samples;
    b.samples = &samples;
    b.sample_min_n = min_n;
    b.list.resize(n);
    std::iota(b.list.begin(), b.list.end(), 0u);
    Node root{};
    root.bounds = bv_empty();
    for (uint32_t i = 0; i < n; ++i) bv_grow(root.bounds, acc(i));
    root.start = 0;
    root.len = n;
    b.nodes.reserve(2 * (size_t)n);
    b.build(root);
    const uint32_t count = std::min<uint32_t>((uint32_t)(samples.size() / 30), capacity);
    std::memcpy(out, samples.data(), sizeof(float) * 30 * (size_t)count);
    return count;
}

// World AABBs of instances as marigold's scene upload computes them
// (marigold/src/app/data/scene/model.rs:191-234): corners (min,min,min),
// (min,min,max), ..., (max,max,max) of the mesh bounds as (x, y, z, 1)
// through the column-major transform; glam 0.30.10's Mat4 * Vec4 (SSE2)
// multiplies each column by the vector's matching component and adds the
// four products in column order, so component r is ((c0 x + c1 y) + c2 z) +
// c3 * 1; Vec3A::min/max are minps/maxps, which return the second operand on
// a tie. out: n x 6 floats. Returns the number of instances whose mesh index
// is out of range (their boxes are left unwritten).
uint32_t oracle_instance_aabbs(const float* mesh_bounds, uint32_t mesh_count, const uint32_t* inst_mesh,
                               const float* xf, uint32_t n, float* out) {
    uint32_t bad = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (inst_mesh[i] >= mesh_count) {
            ++bad;
            continue;
        }
        const float* b = mesh_bounds + 6 * (size_t)inst_mesh[i];
        const float* t = xf + 16 * (size_t)i;
        float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
        for (int c = 0; c < 8; ++c) {
            const float x = b[(c >> 2) & 1 ? 3 : 0], y = b[(c >> 1) & 1 ? 4 : 1], z = b[c & 1 ? 5 : 2];
            for (int r = 0; r < 3; ++r) {
                float v = t[r] * x;
                v = v + t[4 + r] * y;
                v = v + t[8 + r] * z;
                v = v + t[12 + r] * 1.0f;
                lo[r] = lo[r] < v ? lo[r] : v;  // minps(lo, v)
                hi[r] = hi[r] > v ? hi[r] : v;  // maxps(hi, v)
            }
        }
        for (int r = 0; r < 3; ++r) {
            out[6 * (size_t)i + r] = lo[r];
            out[6 * (size_t)i + 3 + r] = hi[r];
        }
    }
    return bad;
}

// Closest hit of each ray against every triangle: the Moller-Trumbore test of
// marigold/assets/shaders/slang/lib/scene.slang:19-89 (|det| < 1e-6 and
// t < 1e-6 reject), every product and sum as written, lowest triangle index
// on equal distances. rays: n_rays x 8 floats (origin xyz, -, dir xyz, -).
void oracle_trace_bruteforce(const float* verts, uint32_t stride_floats, const uint32_t* tris,
                             uint32_t n, const float* rays, uint32_t n_rays, float* out_t,
                             uint32_t* out_prim) {
    for (uint32_t r = 0; r < n_rays; ++r) {
        const float* R = rays + 8 * (size_t)r;
        float best = std::numeric_limits<float>::infinity();
        uint32_t best_prim = 0xFFFFFFFFu;
        for (uint32_t p = 0; p < n; ++p) {
            const float* a = verts + (size_t)tris[3 * (size_t)p] * stride_floats;
            const float* b = verts + (size_t)tris[3 * (size_t)p + 1] * stride_floats;
            const float* c = verts + (size_t)tris[3 * (size_t)p + 2] * stride_floats;
            const float t = moller_trumbore(R[0], R[1], R[2], R[4], R[5], R[6], a, b, c);
            if (t < 0.0f) continue;
            if (t < best || (t == best && p < best_prim)) {
                best = t;
                best_prim = p;
            }
        }
        out_t[r] = best_prim == 0xFFFFFFFFu ? -1.0f : best;
        out_prim[r] = best_prim;
    }
}

// Closest hit of each world-space ray in a two-level scene, by brute force
// (the checker of the two-level traversal; marigold's scene shader,
// scene.slang:91-220, walks the same scene through its TLAS): for every
// instance the ray moves into mesh space through the instance's column-major
// inverse transform, each component ((c0 x + c1 y) + c2 z) + c3 w rounded
// after every product and sum, and meets every triangle of the instance's
// mesh. The hit distance is the ray parameter, the same in both spaces; equal
// distances resolve to the lowest (instance, triangle). meshes: 4 u32 per
// mesh (BLAS root, unused here; triangle offset; triangle count; vertex
// offset); instances: 20 words each (16 floats of the inverse transform, the
// mesh index, 3 unused); tris: vertex index triples relative to the mesh's
// vertex offset.
void oracle_trace_scene_bruteforce(const float* verts, uint32_t stride_floats, const uint32_t* tris,
                                   const uint32_t* meshes, uint32_t n_meshes, const uint32_t* instances,
                                   uint32_t n_inst, const float* rays, uint32_t n_rays, float* out_t,
                                   uint32_t* out_inst, uint32_t* out_tri) {
    auto xform = [](const float* m, float x, float y, float z, float w, float* o) {
        for (int r = 0; r < 3; ++r) {
            float s = m[r] * x;
            s = s + m[4 + r] * y;
            s = s + m[8 + r] * z;
            s = s + m[12 + r] * w;
            o[r] = s;
        }
    };
    for (uint32_t r = 0; r < n_rays; ++r) {
        const float* R = rays + 8 * (size_t)r;
        float best = std::numeric_limits<float>::infinity();
        uint32_t bi = 0xFFFFFFFFu, bp = 0xFFFFFFFFu;
        for (uint32_t k = 0; k < n_inst; ++k) {
            const uint32_t* I = instances + 20 * (size_t)k;
            if (I[16] >= n_meshes) continue;
            float m[16];
            std::memcpy(m, I, sizeof(m));
            const uint32_t* M = meshes + 4 * (size_t)I[16];
            float o[3], d[3];
            xform(m, R[0], R[1], R[2], 1.0f, o);
            xform(m, R[4], R[5], R[6], 0.0f, d);
            for (uint32_t q = 0; q < M[2]; ++q) {
                const uint32_t p = M[1] + q;
                const float* a = verts + (size_t)(tris[3 * (size_t)p] + M[3]) * stride_floats;
                const float* b = verts + (size_t)(tris[3 * (size_t)p + 1] + M[3]) * stride_floats;
                const float* c = verts + (size_t)(tris[3 * (size_t)p + 2] + M[3]) * stride_floats;
                const float t = moller_trumbore(o[0], o[1], o[2], d[0], d[1], d[2], a, b, c);
                if (t < 0.0f) continue;
                if (t < best || (t == best && (k < bi || (k == bi && p < bp)))) {
                    best = t;
                    bi = k;
                    bp = p;
                }
            }
        }
        out_t[r] = bp == 0xFFFFFFFFu ? -1.0f : best;
        out_inst[r] = bi;
        out_tri[r] = bp;
    }
}

}  // extern "C"
