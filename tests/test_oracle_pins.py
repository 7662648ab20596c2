"""More pins of the CPU oracle (no GPU): worked root splits of the
fixed-step adaptive sweep (8 and 16 objects) and of the 32-bin binned sweep
(33 and 64 objects), committed hashes of the oracle's output for the two
single-mesh workloads, and the count of splits that list order decides.

Worked cases. Unit boxes on a line: box i spans [c_i - 0.5, c_i + 0.5] in x
and [0, 1] in y and z, so every centroid is (c_i, 0.5, 0.5). The y and z
centroid extents are 0: the binned sweep returns None there
(bvh/src/lib.rs:339) and the adaptive sweep's thresholds all equal the
minimum, so no object lies strictly below them (:430-437, :306-312). The
root's split is therefore decided on x, where the tables below list every
candidate by hand: its threshold or bin boundary, the objects below it and
the cost (1 + (SA_lt / SA_p) * 8 * n_lt + (SA_gt / SA_p) * 8 * n_gt, :278-288;
SA of a box of x-width w and unit y, z is 2 * (w + w + 1) = 4w + 2).
``root_split`` below restates those rules in float32 numpy, independently
of the C++ oracle, and checks the tables too.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from marigold_b200 import synth
from tests.treecheck import as_words, check_tree

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_hashes.json")
f32 = np.float32


def line_boxes(centroids):
    c = np.asarray(centroids, f32)
    z = np.zeros_like(c)
    return np.stack([c - f32(0.5), z, z, c + f32(0.5), z + f32(1.0), z + f32(1.0)], 1).astype(f32)


def _sa(lo, hi):
    # surface_area, bvh/src/lib.rs:79-91: 2 * ((w*h + w*d) + h*d), one f32 op at a time
    w, h, d = f32(hi[0] - lo[0]), f32(hi[1] - lo[1]), f32(hi[2] - lo[2])
    return f32(f32(2) * f32(f32(f32(w * h) + f32(w * d)) + f32(h * d)))


def _cost(boxes, lt_mask):
    p_lo, p_hi = boxes[:, :3].min(0), boxes[:, 3:].max(0)
    sa_p = _sa(p_lo, p_hi)
    out = f32(1.0)
    for side in (lt_mask, ~lt_mask):
        b = boxes[side]
        term = f32(f32(f32(_sa(b[:, :3].min(0), b[:, 3:].max(0)) / sa_p) * f32(8.0)) * f32(side.sum()))
        out = f32(out + term)
    return out


def root_split(boxes, bins=32):
    """Root split on x of a line of boxes, restated from bvh/src/lib.rs:
    n <= 32 fixed-step adaptive sweep (8 <= n, :428-441) with strict
    `centroid < threshold` (:306-312), else the binned sweep (:331-389);
    first minimum of total_cmp over candidates (:388, :440). Returns
    (candidates, winner): candidates as (threshold or bin index, n_lt, cost)."""
    c = f32(f32(boxes[:, 0] + boxes[:, 3]) * f32(0.5))
    n = c.shape[0]
    cmin, ext = c.min(), f32(c.max() - c.min())
    cands = []
    if n <= 32:
        assert n >= 8
        step = f32(ext / f32(n))  # step_count = len.clamp(8, 32) = n
        for i in range(n):
            thr = f32(cmin + f32(step * f32(f32(i) + f32(0.5))))
            lt = c < thr
            if 0 < lt.sum() < n:
                cands.append((float(thr), int(lt.sum()), float(_cost(boxes, lt))))
    else:
        pct = f32(f32(c - cmin) / ext)
        b = np.minimum(np.floor(f32(pct * f32(bins))).astype(np.int64), bins - 1)  # `as usize`, then min
        for i in range(1, bins):
            lt = b < i
            if 0 < lt.sum() < n:
                cands.append((i, int(lt.sum()), float(_cost(boxes, lt))))
    win = min(range(len(cands)), key=lambda k: (cands[k][2], k))
    return cands, cands[win]


# --- 8 objects: thresholds 0.5 + 2 * (i + 0.5) = 1.5, 3.5, ..., 15.5 (cmin 0.5, ext 16)
# threshold: 1.5  3.5  5.5  7.5  9.5  11.5  13.5  15.5
# n_lt:      1    1    1    1    2    4     7     7      (7.5 and 9.5 are not < themselves)
# SA_p = 4 * 17 + 2 = 70
#   n_lt 1: lt [0, 1]     SA 6,  gt [7, 17]   SA 42 -> 1 + 6/70*8 + 42/70*56  = 35.29
#   n_lt 2: lt [0, 8]     SA 34, gt [9, 17]   SA 34 -> 1 + 34/70*16 + 34/70*48 = 32.09  <- winner
#   n_lt 4: lt [0, 11.5]  SA 48, gt [11, 17]  SA 26 -> 1 + 48/70*32 + 26/70*32 = 34.83
#   n_lt 7: lt [0, 13.5]  SA 56, gt [16, 17]  SA 6  -> 1 + 56/70*56 + 6/70*8   = 46.49
# (thresholds at cmin + step * i would give n_lt 3 for 10.5 (cost 31.40); `<=` would too at 9.5)
EIGHT = [0.5, 7.5, 9.5, 11.0, 11.5, 12.5, 13.0, 16.5]

# --- 16 objects: thresholds 1.5 + 2i = 1.5, 3.5, ..., 31.5 (cmin 0.5, ext 32)
# threshold: 1.5 3.5..11.5 13.5 15.5 17.5 19.5 21.5 23.5 25.5 27.5 29.5 31.5
# n_lt:      1   2         3    3    6    8    9    10   10   12   13   15
# SA_p = 4 * 33 + 2 = 134
#   n_lt 6:  lt [0, 17.5] SA 72, gt [17, 33] SA 66 -> 1 + 72/134*48 + 66/134*80 = 66.19
#   n_lt 8:  lt [0, 19.5] SA 80, gt [20, 33] SA 54 -> 1 + 80/134*64 + 54/134*64 = 65.00  <- winner
#   n_lt 10: lt [0, 22]   SA 90, gt [25, 33] SA 34 -> 1 + 90/134*80 + 34/134*48 = 66.91
SIXTEEN = [0.5, 3.0, 12.5, 15.5, 16.0, 17.0, 17.5, 19.0, 20.5, 21.5, 25.5, 26.5, 29.0, 30.0, 31.0, 32.5]

# --- 33 objects, binned: cmin 0.5, ext 32, so bin = min(floor(c - 0.5), 31); the
# last centroid, 32.5, maps to 32 and saturates into bin 31 with 30.75's neighbour
THIRTY_THREE = [0.5, 1.5, 2.5, 2.75, 3.75, 5.0, 7.25, 8.0, 8.75, 9.25, 11.0, 13.75, 15.5, 16.0, 16.5,
                17.25, 17.5, 18.0, 18.5, 18.75, 19.0, 21.25, 21.75, 22.0, 22.75, 23.0, 24.0, 26.75, 27.0,
                28.75, 30.0, 30.75, 32.5]
THIRTY_THREE_BINS = [0, 1, 2, 2, 3, 4, 6, 7, 8, 8, 10, 13, 15, 15, 16, 16, 17, 17, 18, 18, 18, 20, 21, 21,
                     22, 22, 23, 26, 26, 28, 29, 30, 31]
# candidate i = 14 (bins 0..13: 12 objects, box [0, 14.25]) and i = 15 (bin 14 is
# empty: the same set) tie; the first, i = 14, is taken. SA_p = 4 * 33 + 2 = 134:
#   i = 14: lt [0, 14.25] SA 59, gt [15, 33] SA 74 -> 1 + 59/134*96 + 74/134*168 = 136.04
#   i = 16: lt [0, 16.5]  SA 68, gt [16, 33] SA 70 -> 1 + 68/134*112 + 70/134*152 = 137.24

# --- 64 objects, binned (same grid: bin = min(floor(c - 0.5), 31))
SIXTY_FOUR = [0.5, 1.25, 1.75, 2.5, 4.75, 5.5, 6.25, 6.75, 7.25, 7.75, 8.25, 8.75, 9.0, 9.5, 10.25, 10.75,
              11.0, 11.5, 12.0, 12.5, 13.75, 14.0, 14.5, 15.0, 15.75, 16.0, 16.25, 16.5, 16.75, 17.0, 17.75,
              18.0, 18.5, 19.25, 20.0, 20.5, 20.75, 21.0, 21.25, 22.0, 22.25, 22.5, 22.75, 23.0, 23.75,
              24.25, 25.25, 25.75, 26.25, 26.5, 27.0, 27.5, 28.0, 28.25, 28.75, 29.0, 29.5, 29.75, 30.25,
              30.5, 31.75, 32.0, 32.25, 32.5]
SIXTY_FOUR_BINS = [0, 0, 1, 2, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 13, 13, 14, 14, 15, 15,
                   15, 16, 16, 16, 17, 17, 18, 18, 19, 20, 20, 20, 20, 21, 21, 22, 22, 22, 23, 23, 24, 25,
                   25, 26, 26, 27, 27, 27, 28, 28, 29, 29, 29, 30, 31, 31, 31, 31]
# candidate i = 17 (bins 0..16: 30 objects, box [0, 17.5]) wins:
#   i = 17: lt [0, 17.5] SA 72, gt [17.25, 33] SA 65 -> 1 + 72/134*240 + 65/134*272 = 261.90
#   i = 18: lt [0, 18.5] SA 76, gt [18, 33]    SA 62 -> 1 + 76/134*256 + 62/134*256 = 264.64

CASES = {
    # name: centroids, expected winner (threshold or bin index, n_lt), hand-worked winner cost
    "adaptive_8": (EIGHT, (9.5, 2), 32.086),
    "adaptive_16": (SIXTEEN, (19.5, 8), 65.0),
    "binned_33": (THIRTY_THREE, (14, 12), 136.045),
    "binned_64": (SIXTY_FOUR, (17, 30), 261.896),
}


@pytest.mark.parametrize("name", list(CASES))
def test_worked_root_split(oracle, name):
    cents, (where, n_lt), cost = CASES[name]
    boxes = line_boxes(cents)
    n = boxes.shape[0]
    cands, win = root_split(boxes)
    assert (win[0], win[1]) == (where, n_lt) and abs(win[2] - cost) < 1e-3, win
    if name.startswith("binned"):
        c = np.asarray(cents, f32)
        bins = np.minimum(np.floor(f32(f32(f32(c - c.min()) / f32(c.max() - c.min())) * f32(32))), 31)
        assert bins.astype(int).tolist() == (THIRTY_THREE_BINS if n == 33 else SIXTY_FOUR_BINS)
    r = oracle.build(aabbs=boxes)
    assert r["status"] == 0
    w = as_words(r["nodes"])
    fl = w.view(np.float32)
    lens = r["lens"]
    # root: all objects, children pair at 1; gt child at 1, lt child at 2 (:650-653)
    assert int(w[0, 7]) == 1 and lens[0] == n
    assert lens[2] == n_lt and lens[1] == n - n_lt
    assert int(w[2, 3]) == 0 and int(w[1, 3]) == n_lt  # start indices (:648)
    lt_box = [boxes[:n_lt, 0].min(), 0, 0, boxes[:n_lt, 3].max(), 1, 1]
    gt_box = [boxes[n_lt:, 0].min(), 0, 0, boxes[n_lt:, 3].max(), 1, 1]
    assert fl[2, [0, 1, 2, 4, 5, 6]].tolist() == [float(x) for x in lt_box]
    assert fl[1, [0, 1, 2, 4, 5, 6]].tolist() == [float(x) for x in gt_box]
    # the centroids are sorted, so the lt side is the first n_lt objects
    assert sorted(r["perm"][:n_lt].tolist()) == list(range(n_lt))
    check_tree(r["nodes"], r["lens"], r["perm"], boxes)


def _digest(r):
    h = hashlib.sha256()
    for a in (r["nodes"], r["lens"], r["perm"]):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("key", ["config1_reference", "config1_bins16_adaptive_off", "config2_reference",
                                 "config2_adaptive_steps16"])
def test_oracle_output_hashes(oracle, key):
    g = json.load(open(GOLDEN))[key]
    v, t = synth.config1_mesh() if g["mesh"] == "config1" else synth.config2_mesh()
    r = oracle.build(v, t, root_bounds=synth.mesh_bounds(v), **g["knobs"])
    assert r["status"] == 0 and r["nodes"].shape[0] == g["nodes"]
    assert _digest(r) == g["sha256"]
    # no split of these trees is picked by list order among equal-cost splits
    # over different object sets, so the reference's unstable partitions
    # cannot change them
    assert r["order_dependent"] == g["order_dependent"] == 0
    assert r["tie_events"] == g["tie_events"]


def test_headline_mesh_same_tree_in_both_list_orders(oracle):
    # the two-ended partition_in_place and nth_element order (the reference's
    # algorithmic form) against the stable order: the same bytes
    v, t = synth.config2_mesh()
    b = synth.mesh_bounds(v)
    a = oracle.build(v, t, root_bounds=b)
    f = oracle.build(v, t, root_bounds=b, faithful=True)
    assert _digest(a) == _digest(f)
    assert a["order_dependent"] == f["order_dependent"] == 0
