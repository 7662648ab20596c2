"""CPU checks of the instance-AABB step of marigold's scene upload
(marigold/src/app/data/scene/model.rs:191-234): the oracle's C++ restatement
against the float32 numpy restatement in marigold_b200.synth, and known
answers worked out by hand."""
from __future__ import annotations

import numpy as np

from marigold_b200 import synth


def _random_instances(n, m, seed):
    rng = np.random.default_rng(seed)
    bounds = np.sort(rng.normal(size=(m, 2, 3)).astype(np.float32), axis=1).reshape(m, 6)
    bounds = bounds[:, [0, 1, 2, 3, 4, 5]]
    ids = rng.integers(0, m, n).astype(np.uint32)
    xf = rng.normal(size=(n, 16)).astype(np.float32)
    xf[:, [3, 7, 11]] = 0.0
    xf[:, 15] = 1.0
    return bounds, ids, xf


def test_oracle_matches_numpy_restatement(oracle):
    bounds, ids, xf = _random_instances(5000, 37, 1)
    # signed zeros: zero coordinates and zero matrix entries
    bounds[:3, [0, 3]] = [[-0.0, 0.0], [0.0, 0.0], [-0.0, -0.0]]
    xf[:50, [0, 5]] = 0.0
    xf[50:60, :3] = -0.0
    got, bad = oracle.instance_aabbs(bounds, ids, xf)
    want = synth.instance_aabbs(bounds, ids, xf)
    assert bad == 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_known_answers(oracle):
    bounds = np.array([[1, 2, 3, 4, 6, 8]], np.float32)
    eye = np.eye(4, dtype=np.float32).T.reshape(16)  # column-major identity
    # identity: the mesh bounds
    got, _ = oracle.instance_aabbs(bounds, [0], eye[None])
    assert np.array_equal(got[0], bounds[0])
    # translation by (10, -1, 0.5)
    t = eye.copy()
    t[12:15] = [10, -1, 0.5]
    got, _ = oracle.instance_aabbs(bounds, [0], t[None])
    assert np.array_equal(got[0], np.array([11, 1, 3.5, 14, 5, 8.5], np.float32))
    # mirror x and scale z by 2: min/max swap on x
    s = eye.copy()
    s[0] = -1
    s[10] = 2
    got, _ = oracle.instance_aabbs(bounds, [0], s[None])
    assert np.array_equal(got[0], np.array([-4, 2, 6, -1, 6, 16], np.float32))
    # a quarter turn about z (x -> y, y -> -x)
    r = np.zeros(16, np.float32)
    r[1], r[4], r[10], r[15] = 1, -1, 1, 1
    got, _ = oracle.instance_aabbs(bounds, [0], r[None])
    assert np.array_equal(got[0], np.array([-6, 1, 3, -2, 4, 8], np.float32))


def test_out_of_range_index(oracle):
    bounds, ids, xf = _random_instances(10, 3, 2)
    ids[4] = 3
    _, bad = oracle.instance_aabbs(bounds, ids, xf)
    assert bad == 1


def test_scene_instances_shape():
    ids, xf = synth.scene_instances(3, 20, 100)
    assert ids.shape == (100,) and ids.dtype == np.uint32 and ids.max() < 20
    assert xf.shape == (100, 16) and xf.dtype == np.float32
    assert np.all(xf[:, [3, 7, 11]] == 0) and np.all(xf[:, 15] == 1)
