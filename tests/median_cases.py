"""Inputs that force the reference's median split (bvh/src/lib.rs:444-491,
:527-531) on nodes of more than 1024 objects, where the builder's level
passes run. Shared by the oracle pins (CPU) and the GPU parity tests."""
from __future__ import annotations

import numpy as np


def coincident_boxes(n, seed, center=(0.5, -2.0, 3.0)):
    """n boxes of random half-extents around one centroid: every binned sweep
    refuses (zero centroid extent on all axes), so with MIN_LEAF_OBJECTS = 1
    every node above MAX splits at the median, positionally."""
    rng = np.random.default_rng(seed)
    h = rng.uniform(0.01, 2.0, size=(n, 3)).astype(np.float32)
    c = np.asarray(center, np.float32)
    # centroids (lo + hi) * 0.5 must round to c exactly: symmetric boxes of
    # power-of-two-friendly extents do
    h = np.round(h * 64.0) / 64.0
    return np.concatenate([c - h, c + h], axis=1).astype(np.float32)


def outlier_boxes(n, seed, outliers=1):
    """Distinct centroids where, with MIN_LEAF_OBJECTS >= 2, no binned
    candidate keeps MIN objects on both sides: `outliers` objects sit at the
    low end of every axis and the rest crowd into the top bin. Small random
    extents give every axis a different median cost."""
    rng = np.random.default_rng(seed)
    c = np.empty((n, 3), np.float32)
    c[:outliers] = rng.uniform(0.0, 0.001, size=(outliers, 3))
    c[outliers:] = rng.uniform(0.995, 1.0, size=(n - outliers, 3))
    perm = rng.permutation(n)
    c = c[perm]
    h = rng.uniform(0.0005, 0.02, size=(n, 3)).astype(np.float32)
    lo = (c - h).astype(np.float32)
    hi = (c + h).astype(np.float32)
    return np.concatenate([lo, hi], axis=1)


def cluster_in_mesh(n_random, n_cluster, seed):
    """Random boxes plus a cluster of n_cluster copies of one box: deep in the
    tree a node of only the cluster's copies needs the median."""
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-10, 10, size=(n_random, 3)).astype(np.float32)
    ext = rng.uniform(0.01, 0.5, size=(n_random, 3)).astype(np.float32)
    boxes = np.concatenate([lo, lo + ext], axis=1)
    one = np.array([[1.0, 2.0, 3.0, 1.5, 2.25, 3.125]], np.float32)
    allb = np.concatenate([boxes, np.repeat(one, n_cluster, axis=0)], axis=0)
    return allb[rng.permutation(allb.shape[0])]
