"""Forced median splits on nodes above the subtree-CTA size (needs a B200).

The reference forces a median when every binned sweep of a node refuses and
the node holds more than MAX_LEAF_OBJECTS objects (bvh/src/lib.rs:527-531,
median_split :444-491, run on axes 0, 1, 2 over the same list). On the GPU
such nodes above medium_max objects are split by the median passes after the
pipeline. Every case here equals the oracle word for word (nodes, lengths,
permutation) and agrees with it on the status, including the reference's
containment assertion failing after a median whose winning axis is not 2.
"""
import ctypes

import numpy as np
import pytest

from marigold_b200 import BvhSettings, _lib, build_batch_device, synth
from tests import median_cases as mc
from tests.gpuhelp import gpu_build
from tests.treecheck import check_tree, compare_exact

pytestmark = pytest.mark.gpu


def both(oracle, ctx, **kw):
    o = oracle.build(**kw)
    g = gpu_build(ctx, **kw)
    assert g["status"] == o["status"], (g["status"], g["error"], o["status"])
    if o["status"] >= 0:
        msg = compare_exact(g["nodes"], g["lens"], g["perm"], o["nodes"], o["lens"], o["perm"])
        assert msg is None, msg
        assert g["stats"]["median_splits"] == o["stats"]["median_splits"]
    return o, g


@pytest.mark.parametrize("n", [1025, 1030, 2048, 2049, 5000, 40000])
def test_coincident_centroids(oracle, gpu_ctx, n):
    boxes = mc.coincident_boxes(n, n)
    o, g = both(oracle, gpu_ctx, aabbs=boxes)
    assert o["stats"]["median_splits"] == n - 1
    check_tree(g["nodes"], g["lens"], g["perm"], boxes)


@pytest.mark.parametrize("n,seed,kw", [
    (5000, 3, dict(min_leaf=2, max_leaf=4)),
    (20000, 4, dict(min_leaf=2, max_leaf=4)),
    (5000, 5, dict(min_leaf=3, max_leaf=8)),
    (3000, 6, dict(min_leaf=2, max_leaf=2)),
    (70000, 7, dict(min_leaf=2, max_leaf=4)),
])
def test_distinct_keys_min_leaf(oracle, gpu_ctx, n, seed, kw):
    boxes = mc.outlier_boxes(n, seed, outliers=1 if kw["min_leaf"] == 2 else 2)
    o, g = both(oracle, gpu_ctx, aabbs=boxes, **kw)
    # MIN = MAX = 2 (seed 6) ends in the reference's containment assertion
    assert o["stats"]["median_splits"] > 0 or o["status"] == -5


@pytest.mark.parametrize("kw", [dict(), dict(max_leaf=4), dict(max_depth=6), dict(min_leaf=2, max_leaf=3)])
def test_cluster_inside_mesh(oracle, gpu_ctx, kw):
    boxes = mc.cluster_in_mesh(20000, 3000, 6)
    both(oracle, gpu_ctx, aabbs=boxes, **kw)


def test_median_assertion_reported(oracle, gpu_ctx):
    # axis-2 halves whose centroids leave the winning axis's boxes: the
    # reference panics at bvh/src/lib.rs:637-646; both report the assertion
    rng = np.random.default_rng(1)
    n = 3000
    t = rng.uniform(0, 1, n).astype(np.float32)
    c = np.stack([0.995 + 0.005 * t, rng.uniform(0.995, 1.0, n), 1.0 - 0.005 * t], 1).astype(np.float32)
    c[0] = 0.0
    h = np.array([0.0001, 0.01, 0.01], np.float32)
    boxes = np.concatenate([c - h, c + h], 1).astype(np.float32)
    o, g = both(oracle, gpu_ctx, aabbs=boxes, min_leaf=2, max_leaf=4)
    assert o["status"] == -5


def test_level_pass_median_at_tuned_switch_over(oracle):
    # with medium_max 512, nodes of 513..1024 objects take the level passes
    ctx = _lib.Context(0)
    ctx.check(ctx.L.mgbvh_set_tuning(ctx.ptr, 512))
    for n in (600, 1024, 3000):
        both(oracle, ctx, aabbs=mc.coincident_boxes(n, 11 + n))
        both(oracle, ctx, aabbs=mc.outlier_boxes(n, n), min_leaf=2, max_leaf=4)
    ctx.close()


def test_triangles_with_duplicates_above_cta_size(oracle, gpu_ctx):
    # a mesh whose triangles repeat 1500 times: a node of the copies alone
    v, t = synth.random_triangles(4000, 21)
    t = np.concatenate([t, np.repeat(t[:1], 1500, axis=0)], axis=0)
    both(oracle, gpu_ctx, vertices=v, triangles=t, root_bounds=synth.mesh_bounds(v))


def test_streamed_host_output_with_medians(oracle, gpu_ctx):
    # page-locked outputs: node chunks stream during the pipeline, so the
    # median subtrees built afterwards must reach the caller's array too
    from tests.test_gpu_stream_out import host_build
    boxes = mc.cluster_in_mesh(30000, 4000, 8)
    o = oracle.build(aabbs=boxes)
    for pinned in (True, False):
        r = host_build(gpu_ctx, aabbs=boxes, pinned=pinned)
        msg = compare_exact(r["nodes"], r["lens"], r["perm"], o["nodes"], o["lens"], o["perm"])
        assert msg is None, (pinned, msg)


def _batch(ctx, descs, slots, total, stream=None, **kw):
    import torch
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(total, dtype=torch.int32, device="cuda")
    offs, rc, st = build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens, stream=stream,
                                      **kw)
    torch.cuda.synchronize()
    return (offs, rc, st, nodes.cpu().numpy().view(np.uint32).reshape(-1, 8),
            lens.cpu().numpy().view(np.uint32), perm.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("graph", [False, True])
def test_batched_build_with_medians(oracle, graph):
    import torch
    v, t = synth.random_triangles(3000, 31)
    objs = [("tri", v, t), ("aabb", mc.coincident_boxes(5000, 32), None),
            ("aabb", mc.cluster_in_mesh(8000, 2000, 33), None)]
    descs = []
    for kind, a, b in objs:
        if kind == "tri":
            descs.append({"vertices": torch.from_numpy(a).cuda(),
                          "triangles": torch.from_numpy(b.view(np.int32)).cuda()})
        else:
            descs.append({"aabbs": torch.from_numpy(a).cuda()})
    sizes = [b.shape[0] if k == "tri" else a.shape[0] for k, a, b in objs]
    slots = sum(2 * n - 1 for n in sizes)
    ctx = _lib.Context(0)
    stream = torch.cuda.Stream()
    if graph:
        ctx.check(ctx.L.mgbvh_set_graph_capture(ctx.ptr, 1))
    for rep in range(3 if graph else 1):
        offs, rc, st, nodes, lens, perm = _batch(ctx, descs, slots, sum(sizes), stream=stream)
        assert rc >= 0
        assert st["graph_replay"] == 0  # a batch that needs medians is never replayed from a graph
        first = 0
        for m, (kind, a, b) in enumerate(objs):
            o = oracle.build(a, b) if kind == "tri" else oracle.build(aabbs=a)
            n = sizes[m]
            msg = compare_exact(nodes[offs[m]:offs[m + 1]], lens[offs[m]:offs[m + 1]], perm[first:first + n],
                                o["nodes"], o["lens"], o["perm"])
            assert msg is None, (rep, m, msg)
            first += n
    ctx.close()
