"""CUDA builder vs the CPU oracle, bit for bit (needs a B200).

Every case builds the same seeded input with the oracle (stable parity mode)
and with libmgbvh.so through the C ABI, and compares node words, per-node
object counts and the permutation exactly. Structural invariants of the
reference (treecheck.check_tree) are checked on the GPU result as well.
"""
import numpy as np
import pytest

from marigold_b200 import _lib, synth
from tests.gpuhelp import gpu_build
from tests.treecheck import check_tree, compare_exact

pytestmark = pytest.mark.gpu


def unit_box(x, y=0.0, z=0.0):
    return [x, y, z, x + 1.0, y + 1.0, z + 1.0]


def both(oracle, ctx, **kw):
    o = oracle.build(**kw)
    g = gpu_build(ctx, **kw)
    assert g["status"] == o["status"], (g["status"], g["error"], o["status"])
    msg = compare_exact(g["nodes"], g["lens"], g["perm"], o["nodes"], o["lens"], o["perm"])
    assert msg is None, msg
    return o, g


KNOWN = [
    [unit_box(0)],
    [unit_box(0), unit_box(2)],
    [unit_box(2), unit_box(0)],
    [unit_box(0), unit_box(2), unit_box(4), unit_box(6)],
    [unit_box(0)] * 4,
    [unit_box(0)] * 40,      # forced medians through the medium-node path
    [unit_box(0)] * 1030,    # coincident centroids in a node above the CTA size: level-pass medians
]


@pytest.mark.parametrize("case", range(len(KNOWN)))
def test_known_answer_cases(oracle, gpu_ctx, case):
    boxes = np.array(KNOWN[case], np.float32)
    both(oracle, gpu_ctx, aabbs=boxes)


def test_depth_cap_known_answer(oracle, gpu_ctx):
    boxes = np.array([unit_box(0), unit_box(2), unit_box(4), unit_box(6)], np.float32)
    o, g = both(oracle, gpu_ctx, aabbs=boxes, max_depth=1)
    assert g["stats"]["depth_capped_leaves"] == 2 and g["nodes"].shape[0] == 3


@pytest.mark.parametrize("n", [2, 3, 5, 7, 8, 9, 16, 31, 32, 33, 34, 63, 64, 100, 500, 1000, 1023,
                               1024, 1025, 1026, 2047, 2048, 2049, 4096, 5000, 20000])
def test_random_sizes(oracle, gpu_ctx, n):
    v, t = synth.random_triangles(n, 100 + n)
    b = synth.mesh_bounds(v)
    o, g = both(oracle, gpu_ctx, vertices=v, triangles=t, root_bounds=b)
    check_tree(g["nodes"], g["lens"], g["perm"], synth.triangle_aabbs(v, t), root_bounds=b)


@pytest.mark.parametrize("kw", [
    dict(max_depth=0), dict(max_depth=1), dict(max_depth=3), dict(max_depth=8), dict(max_depth=12),
    dict(min_leaf=2, max_leaf=4), dict(min_leaf=1, max_leaf=8), dict(min_leaf=4, max_leaf=4),
    dict(min_leaf=3, max_leaf=16), dict(min_leaf=1, max_leaf=2000),
    dict(bins=16, adaptive_max_n=0), dict(bins=16), dict(bins=8), dict(bins=2), dict(bins=31),
    dict(adaptive_steps=16), dict(adaptive_steps=1), dict(adaptive_max_n=8), dict(adaptive_max_n=1),
    dict(adaptive_max_n=0), dict(bins=12, adaptive_steps=5, adaptive_max_n=20),
])
def test_knobs_and_leaf_bounds(oracle, gpu_ctx, kw):
    v, t = synth.random_triangles(6000, 7)
    both(oracle, gpu_ctx, vertices=v, triangles=t, **kw)


@pytest.mark.parametrize("small_threads,small_warps", [(256, 16), (256, 24), (128, 16), (64, 24)])
@pytest.mark.parametrize("kw", [dict(), dict(bins=16)])
def test_launch_shapes_leave_the_tree_unchanged(oracle, small_threads, small_warps, kw):
    # the small-subtree kernel's block size and occupancy (both register
    # budgets, level-synchronous and depth-first builders) change speed only
    v, t = synth.random_triangles(20000, 11)
    ctx = _lib.Context(0)
    try:
        ctx.set_launch_shape(small_threads, 0)
        ctx.set_small_occupancy(small_warps)
        both(oracle, ctx, vertices=v, triangles=t, **kw)
    finally:
        ctx.close()


def test_small_occupancy_rejects_other_values(gpu_ctx):
    for bad in (8, 20, 32):
        assert gpu_ctx.L.mgbvh_set_small_occupancy(gpu_ctx.ptr, bad) == _lib.ERR_UNSUPPORTED
    assert gpu_ctx.L.mgbvh_set_small_occupancy(gpu_ctx.ptr, 0) == 0


def test_aabb_path_tlas_like(oracle, gpu_ctx):
    # the TLAS path: AsBoundingVolume objects, root bounds = union (bounds: None)
    rng = np.random.default_rng(3)
    lo = rng.uniform(-100, 100, size=(4096, 3)).astype(np.float32)
    ext = rng.uniform(0.5, 20, size=(4096, 3)).astype(np.float32)
    boxes = np.concatenate([lo, lo + ext], axis=1)
    o, g = both(oracle, gpu_ctx, aabbs=boxes)
    check_tree(g["nodes"], g["lens"], g["perm"], boxes)


def test_duplicates_and_clusters(oracle, gpu_ctx):
    # many exactly duplicated triangles: coincident centroids below the CTA size
    v, t = synth.random_triangles(300, 9)
    t = np.concatenate([t] * 3 + [t[:7]] * 5, axis=0)
    both(oracle, gpu_ctx, vertices=v, triangles=t)


def test_config1_reference_profile(oracle, gpu_ctx):
    v, t = synth.config1_mesh()
    b = synth.mesh_bounds(v)
    o, g = both(oracle, gpu_ctx, vertices=v, triangles=t, root_bounds=b)
    assert g["nodes"].shape[0] == 2 * 65536 - 1
    for k in ("node_count", "leaf_node_count", "height", "min_leaf_object_count",
              "max_leaf_object_count"):
        assert g["stats"][k] == o["stats"][k], k


def test_config1_sixteen_bins_adaptive_off(oracle, gpu_ctx):
    v, t = synth.config1_mesh()
    both(oracle, gpu_ctx, vertices=v, triangles=t, root_bounds=synth.mesh_bounds(v), bins=16,
         adaptive_max_n=0)


def test_config2_reference_profile(oracle, gpu_ctx):
    v, t = synth.config2_mesh()
    b = synth.mesh_bounds(v)
    o, g = both(oracle, gpu_ctx, vertices=v, triangles=t, root_bounds=b)
    check_tree(g["nodes"], g["lens"], g["perm"], synth.triangle_aabbs(v, t), root_bounds=b)


def test_config2_thirtytwo_bins_sixteen_thresholds(oracle, gpu_ctx):
    v, t = synth.config2_mesh()
    both(oracle, gpu_ctx, vertices=v, triangles=t, root_bounds=synth.mesh_bounds(v), bins=32,
         adaptive_steps=16)


def test_bad_index_is_an_error(gpu_ctx):
    v, t = synth.random_triangles(100, 1)
    t = t.copy()
    t[50, 1] = v.shape[0] + 5
    g = gpu_build(gpu_ctx, vertices=v, triangles=t)
    assert g["status"] == -1 and "index" in g["error"]


def test_capacity_too_small_is_an_error(gpu_ctx):
    v, t = synth.random_triangles(100, 1)
    g = gpu_build(gpu_ctx, vertices=v, triangles=t, capacity=150)
    assert g["status"] == -2


def test_empty_input_warns(gpu_ctx):
    g = gpu_build(gpu_ctx, aabbs=np.zeros((0, 6), np.float32))
    assert g["status"] == 1 and g["nodes"].shape[0] == 0


def test_repeated_builds_on_one_context(oracle, gpu_ctx):
    # scratch reuse across sizes must not leak state between builds
    for n in (5000, 100, 70000, 33, 5000):
        v, t = synth.random_triangles(n, 500 + n)
        both(oracle, gpu_ctx, vertices=v, triangles=t)


def test_device_entry_point_matches_host_entry_point(oracle, gpu_ctx):
    import torch
    from marigold_b200 import BvhSettings, build_device
    v, t = synth.random_triangles(40000, 77)
    o = oracle.build(v, t)
    dv = torch.from_numpy(v).cuda()
    dt = torch.from_numpy(t.astype(np.int32)).cuda()
    n = t.shape[0]
    nodes = torch.zeros((2 * n - 1) * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(2 * n - 1, dtype=torch.int32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    count, rc, st = build_device(gpu_ctx, BvhSettings(), nodes, perm, vertices=dv, triangles=dt,
                                 out_lens=lens)
    torch.cuda.synchronize()
    assert rc == 0 and count == 2 * n - 1
    gw = nodes.cpu().numpy().view(np.uint32).reshape(-1, 8)
    msg = compare_exact(gw, lens.cpu().numpy().view(np.uint32), perm.cpu().numpy().view(np.uint32),
                        o["nodes"], o["lens"], o["perm"])
    assert msg is None, msg


def test_level_hint_across_meshes(oracle):
    """A context launches the level passes its previous build needed without
    reading counts in between; a deeper tree than the hint is rebuilt with
    counts read, a shallower one runs empty passes. Every tree equals the
    oracle's."""
    from marigold_b200 import synth as _synth
    ctx = _lib.Context(0)
    try:
        small = _synth.random_triangles(5000, seed=71)
        large = _synth.random_triangles(200000, seed=72)
        for v, t in (small, large, large, small, large):
            g = gpu_build(ctx, v, t)
            o = oracle.build(v, t)
            assert g["status"] == o["status"] == 0
            assert compare_exact(g["nodes"], g["lens"], g["perm"], o["nodes"], o["lens"], o["perm"]) is None
    finally:
        ctx.close()


@pytest.mark.parametrize("key", ["config1_reference", "config1_bins16_adaptive_off", "config2_reference",
                                 "config2_adaptive_steps16"])
def test_output_hashes_equal_the_committed_oracle_hashes(gpu_ctx, key):
    # tests/golden/oracle_hashes.json holds the oracle's bytes for these
    # workloads (tests/golden/make_oracle_hashes.py); no oracle run here
    import hashlib
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_hashes.json")))[key]
    v, t = synth.config1_mesh() if g["mesh"] == "config1" else synth.config2_mesh()
    r = gpu_build(gpu_ctx, vertices=v, triangles=t, root_bounds=synth.mesh_bounds(v), **g["knobs"])
    assert r["status"] == 0 and r["nodes"].shape[0] == g["nodes"]
    h = hashlib.sha256()
    for a in (r["nodes"], r["lens"], r["perm"]):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    assert h.hexdigest() == g["sha256"]


@pytest.mark.parametrize("name", ["adaptive_8", "adaptive_16", "binned_33", "binned_64"])
def test_worked_root_splits(oracle, gpu_ctx, name):
    from tests.test_oracle_pins import CASES, line_boxes
    boxes = line_boxes(CASES[name][0])
    both(oracle, gpu_ctx, aabbs=boxes)
    # the same lines with 16 bins and 4 fixed adaptive steps
    both(oracle, gpu_ctx, aabbs=boxes, bins=16, adaptive_steps=4)
