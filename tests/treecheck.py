"""Structural checks on a built tree: the reference's own invariants.

bvh/src/lib.rs asserts, in release builds, that both children of a split are
non-empty and hold the counts the split promised (:618-634), that every
child's bounds contain the centroids of its objects (:637-646), that leaf
sizes obey MIN/MAX when feasible (:823-827) and that a <1,1> tree has exactly
2N-1 nodes (:831-834). The node numbering is a pre-order over child pairs,
gt child first (:650-663).
"""
from __future__ import annotations

import numpy as np


def as_words(nodes) -> np.ndarray:
    a = np.ascontiguousarray(nodes)
    return a.view(np.uint32).reshape(-1, 8)


def check_tree(nodes, lens, perm, aabbs, *, min_leaf=1, max_leaf=1, max_depth=32,
               root_bounds=None, exact_bounds=True):
    w = as_words(nodes)
    lens = np.asarray(lens, dtype=np.int64)
    count = w.shape[0]
    n = aabbs.shape[0]
    assert count >= 1
    assert np.array_equal(np.sort(perm), np.arange(n)), "permutation is not a bijection"
    f = w.view(np.float32)
    bmin, bmax = f[:, 0:3], f[:, 4:7]
    start = w[:, 3].astype(np.int64)
    child = w[:, 7].astype(np.int64)
    boxes = aabbs[perm]  # objects in final order
    cent = (boxes[:, 0:3] + boxes[:, 3:6]) * np.float32(0.5)
    assert start[0] == 0 and lens[0] == n
    if root_bounds is not None:
        assert np.array_equal(f[0, [0, 1, 2, 4, 5, 6]], np.asarray(root_bounds, np.float32))
    # pre-order numbering (gt first) and reachability
    nxt = 1
    stack = [(0, 0)]
    visited = np.zeros(count, dtype=bool)
    leaf_sizes = []
    max_seen = 0
    while stack:
        i, d = stack.pop()
        assert not visited[i]
        visited[i] = True
        max_seen = max(max_seen, d)
        assert d <= max_depth
        if child[i] == 0:
            leaf_sizes.append(lens[i])
            continue
        c = child[i]
        assert c == nxt, f"node {i}: child {c}, pre-order expects {nxt}"
        nxt += 2
        gt, lt = c, c + 1
        assert lens[gt] > 0 and lens[lt] > 0
        assert lens[gt] + lens[lt] == lens[i]
        assert start[lt] == start[i] and start[gt] == start[i] + lens[lt]
        stack.append((lt, d + 1))
        stack.append((gt, d + 1))
    assert nxt == count and visited.all()
    # containment of centroids, and bounds = union of the objects (vectorised)
    for i in range(1, count):
        s, l = start[i], lens[i]
        c = cent[s:s + l]
        assert (c >= bmin[i]).all() and (c <= bmax[i]).all(), f"node {i} misses a centroid"
        if exact_bounds:
            b = boxes[s:s + l]
            assert np.array_equal(b[:, 0:3].min(axis=0), bmin[i]), f"node {i} min"
            assert np.array_equal(b[:, 3:6].max(axis=0), bmax[i]), f"node {i} max"
    leaf_sizes = np.asarray(leaf_sizes)
    if min_leaf == 1 and max_leaf == 1 and max_seen < max_depth:
        assert count == 2 * n - 1
    return {"count": count, "leaves": len(leaf_sizes), "height_seen": max_seen}


def compare_exact(a_nodes, a_lens, a_perm, b_nodes, b_lens, b_perm):
    """Bit-exact comparison of two builds; returns None or a message."""
    aw, bw = as_words(a_nodes), as_words(b_nodes)
    if aw.shape != bw.shape:
        return f"node count {aw.shape[0]} vs {bw.shape[0]}"
    bad = np.nonzero((aw != bw).any(axis=1))[0]
    if bad.size:
        i = bad[0]
        return f"{bad.size} nodes differ, first {i}: {aw[i].tolist()} vs {bw[i].tolist()}"
    if not np.array_equal(np.asarray(a_lens), np.asarray(b_lens)):
        return "lens differ"
    if not np.array_equal(np.asarray(a_perm), np.asarray(b_perm)):
        k = np.nonzero(np.asarray(a_perm) != np.asarray(b_perm))[0]
        return f"{k.size} permutation entries differ, first at {k[0]}"
    return None
