"""Pins of the CPU oracle (no GPU).

The reference ships no tests or golden vectors for its builder, so the oracle
is pinned three ways: (1) hand-worked known-answer trees, derived on paper
from bvh/src/lib.rs for tiny inputs; (2) the reference's own release-mode
invariants on seeded inputs; (3) its two list-order modes (stable parity
mode, and the reference's two-ended partition + nth_element) agreeing on the
tree wherever the reference's result does not depend on list order.
"""
import numpy as np
import pytest

from marigold_b200 import synth
from tests.treecheck import as_words, check_tree


def unit_box(x, y=0.0, z=0.0):
    return [x, y, z, x + 1.0, y + 1.0, z + 1.0]


def node_rows(res):
    w = as_words(res["nodes"])
    f = w.view(np.float32)
    return [(tuple(f[i, 0:3]), int(w[i, 3]), tuple(f[i, 4:7]), int(w[i, 7]), int(res["lens"][i]))
            for i in range(w.shape[0])]


def test_single_object_is_a_leaf(oracle):
    r = oracle.build(aabbs=np.array([unit_box(0)], np.float32))
    assert r["status"] == 0
    assert node_rows(r) == [((0, 0, 0), 0, (1, 1, 1), 0, 1)]
    assert r["perm"].tolist() == [0]
    assert r["stats"]["leaf_node_count"] == 0  # leaves are counted from nodes[1..] (:769-773)


def test_empty_list_warns(oracle):
    r = oracle.build(aabbs=np.zeros((0, 6), np.float32))
    assert r["status"] == 1 and r["nodes"].shape[0] == 0


def test_two_boxes_known_answer(oracle):
    # n = 2 -> adaptive sweep with each centroid as threshold (:417-427).
    # axis 0: thr 0.5 gives an empty lt side (refused by MIN = 1); thr 2.5
    # splits {obj0} | {obj1}. Axes 1 and 2 have equal centroids -> refused.
    r = oracle.build(aabbs=np.array([unit_box(0), unit_box(2)], np.float32))
    assert node_rows(r) == [
        ((0, 0, 0), 0, (3, 1, 1), 1, 2),
        ((2, 0, 0), 1, (3, 1, 1), 0, 1),  # gt child first (:652)
        ((0, 0, 0), 0, (1, 1, 1), 0, 1),  # lt child at child_node + 1
    ]
    assert r["perm"].tolist() == [0, 1]


def test_two_boxes_reversed_known_answer(oracle):
    r = oracle.build(aabbs=np.array([unit_box(2), unit_box(0)], np.float32))
    assert node_rows(r) == [
        ((0, 0, 0), 0, (3, 1, 1), 1, 2),
        ((2, 0, 0), 1, (3, 1, 1), 0, 1),
        ((0, 0, 0), 0, (1, 1, 1), 0, 1),
    ]
    assert r["perm"].tolist() == [1, 0]  # the list is permuted in place


def test_four_in_a_row_depth_cap_known_answer(oracle):
    # centroids x = 0.5, 2.5, 4.5, 6.5: thresholds 2.5 / 6.5 cost 1 + 1.6 + 17.6,
    # threshold 4.5 costs 1 + 2 * (14/30) * 8 * 2 ~ 15.93 -> split {0,1} | {2,3};
    # max_depth 1 turns both children into two-object leaves (:556).
    boxes = np.array([unit_box(0), unit_box(2), unit_box(4), unit_box(6)], np.float32)
    r = oracle.build(aabbs=boxes, max_depth=1)
    assert node_rows(r) == [
        ((0, 0, 0), 0, (7, 1, 1), 1, 4),
        ((4, 0, 0), 2, (7, 1, 1), 0, 2),
        ((0, 0, 0), 0, (3, 1, 1), 0, 2),
    ]
    assert r["stats"]["depth_capped_leaves"] == 2
    assert r["stats"]["height"] == 0


def test_four_in_a_row_full_tree_known_answer(oracle):
    boxes = np.array([unit_box(0), unit_box(2), unit_box(4), unit_box(6)], np.float32)
    r = oracle.build(aabbs=boxes)
    # pre-order over pairs, gt first: root -> (gt {2,3} at 1, lt {0,1} at 2);
    # node 1 -> children 3 (obj 3), 4 (obj 2); node 2 -> children 5 (obj 1), 6 (obj 0)
    assert node_rows(r) == [
        ((0, 0, 0), 0, (7, 1, 1), 1, 4),
        ((4, 0, 0), 2, (7, 1, 1), 3, 2),
        ((0, 0, 0), 0, (3, 1, 1), 5, 2),
        ((6, 0, 0), 3, (7, 1, 1), 0, 1),
        ((4, 0, 0), 2, (5, 1, 1), 0, 1),
        ((2, 0, 0), 1, (3, 1, 1), 0, 1),
        ((0, 0, 0), 0, (1, 1, 1), 0, 1),
    ]
    assert r["perm"].tolist() == [0, 1, 2, 3]
    assert r["stats"]["height"] == 1


def test_coincident_centroids_force_median_known_answer(oracle):
    # four identical boxes: every threshold leaves one side empty on every
    # axis, so the median split is forced (:527-531) at index n/2.
    boxes = np.array([unit_box(0)] * 4, np.float32)
    r = oracle.build(aabbs=boxes)
    assert [(row[1], row[3], row[4]) for row in node_rows(r)] == [
        (0, 1, 4), (2, 3, 2), (0, 5, 2), (3, 0, 1), (2, 0, 1), (1, 0, 1), (0, 0, 1)]
    assert r["stats"]["median_splits"] == 3
    assert r["perm"].tolist() == [0, 1, 2, 3]


def test_settings_bounds_are_the_root_bounds(oracle):
    boxes = np.array([unit_box(0), unit_box(2)], np.float32)
    rb = np.array([-1, -1, -1, 5, 5, 5], np.float32)
    r = oracle.build(aabbs=boxes, root_bounds=rb)
    f = as_words(r["nodes"]).view(np.float32)
    assert f[0, [0, 1, 2, 4, 5, 6]].tolist() == rb.tolist()


def test_triangle_aabb_is_min_max_of_three_vertices(oracle):
    # MeshTriangle::bounding_volume (mesh_interface/src/lib.rs:19-30)
    v = np.zeros((3, 8), np.float32)
    v[0, :3] = [1, 5, -2]
    v[1, :3] = [3, -1, 0]
    v[2, :3] = [0, 2, 4]
    r = oracle.build(v, np.array([[0, 1, 2]], np.uint32))
    f = as_words(r["nodes"]).view(np.float32)
    assert f[0, [0, 1, 2, 4, 5, 6]].tolist() == [0, -1, -2, 3, 5, 4]


@pytest.mark.parametrize("n,seed", [(3, 1), (7, 2), (8, 3), (31, 4), (32, 5), (33, 6), (100, 7),
                                    (1000, 8), (5000, 9)])
def test_invariants_random(oracle, n, seed):
    v, t = synth.random_triangles(n, seed)
    b = synth.mesh_bounds(v)
    r = oracle.build(v, t, root_bounds=b)
    assert r["status"] == 0
    check_tree(r["nodes"], r["lens"], r["perm"], synth.triangle_aabbs(v, t), root_bounds=b)


@pytest.mark.parametrize("kw", [dict(max_depth=5), dict(min_leaf=2, max_leaf=4),
                                dict(min_leaf=1, max_leaf=8), dict(bins=16, adaptive_max_n=0),
                                dict(adaptive_steps=16), dict(bins=8), dict(adaptive_max_n=8)])
def test_invariants_knobs(oracle, kw):
    v, t = synth.random_triangles(3000, 11)
    r = oracle.build(v, t, **kw)
    assert r["status"] in (0, 2)
    check_tree(r["nodes"], r["lens"], r["perm"], synth.triangle_aabbs(v, t),
               min_leaf=kw.get("min_leaf", 1), max_leaf=kw.get("max_leaf", 1),
               max_depth=kw.get("max_depth", 32))


@pytest.mark.parametrize("n,seed", [(2000, 21), (20000, 22)])
def test_stable_and_faithful_modes_agree(oracle, n, seed):
    # with single-object leaves and no ties the tree fixes the permutation,
    # so the reference's unstable partitions and the stable ones coincide
    v, t = synth.random_triangles(n, seed)
    a = oracle.build(v, t)
    b = oracle.build(v, t, faithful=True)
    assert a["tie_events"] == 0
    assert np.array_equal(a["nodes"], b["nodes"]) and np.array_equal(a["perm"], b["perm"])


def test_icosphere_small_is_consistent(oracle):
    v, t = synth.noisy_icosphere(3, seed=5)
    assert v.shape[0] == 10 * 4 ** 3 + 2 and t.shape[0] == 20 * 4 ** 3
    r = oracle.build(v, t, root_bounds=synth.mesh_bounds(v))
    check_tree(r["nodes"], r["lens"], r["perm"], synth.triangle_aabbs(v, t))
