"""glTF ingestion (marigold_b200.gltf, the reference's gltf_loading crate):
accessor reading, primitive filtering, vertex records, bounds, scene graph
transforms and the packed mesh numbering, on scenes the tests write."""
from __future__ import annotations

import logging

import numpy as np
import pytest

from marigold_b200 import gltf
from tests import gltf_files


def _quad():
    v = np.zeros((4, 8), np.float32)
    v[:, 0:3] = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]]
    v[:, 4:7] = [0, 0, 1]
    v[:, 3] = [0.0, 1.0, 1.0, 128 / 255]
    v[:, 7] = [0.0, 0.0, 1.0, 1.0]
    return v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


def _scene(tmp_path, form):
    buf = gltf_files.buffer()
    qv, qt = _quad()
    rng = np.random.default_rng(3)
    bv = np.zeros((5, 8), np.float32)
    bv[:, 0:3] = rng.normal(size=(5, 3))
    bv[:, 4:7] = [1, 0, 0]
    bv[:, 3] = rng.random(5)
    bv[:, 7] = rng.random(5)
    bt = np.array([[0, 1, 2], [2, 3, 4]], np.uint32)
    p00 = gltf_files.mesh_primitive(buf, qv, qt, uv_u8=True, index_type=5123)
    p01 = dict(p00, mode=1)  # lines: not a triangle primitive
    p10 = gltf_files.mesh_primitive(buf, bv, bt, interleaved=True, index_type=5125, extra_indices=1)
    rot_z = [0, -1, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 5, 6, 7, 1]  # column-major: x -> -y, y -> x, then (5,6,7)
    doc = {
        "meshes": [{"primitives": [p00, p01]}, {"primitives": [p10]}],
        "nodes": [
            {"translation": [1, 2, 3], "scale": [2, 2, 2], "children": [1]},
            {"matrix": rot_z, "mesh": 0},
            {"mesh": 1},
            {"scale": [1, 2, 1], "mesh": 1},
        ],
        "scenes": [{"name": "main", "nodes": [0, 2]}, {"nodes": [3]}],
    }
    return gltf_files.write(str(tmp_path / form), doc, buf, form), (qv, qt, bv, bt, rot_z)


@pytest.mark.parametrize("form", ["gltf", "glb", "data"])
def test_load_scene(tmp_path, caplog, form):
    path, (qv, qt, bv, bt, rot_z) = _scene(tmp_path, form)
    with caplog.at_level(logging.WARNING, logger="marigold_b200.gltf"):
        sc = gltf.GltfScenes.load(path)
    assert sorted(sc.meshes) == [(0, 0), (1, 0)]  # the lines primitive is dropped
    q = sc.meshes[(0, 0)]
    assert q.vertices.dtype == np.float32 and q.vertices.shape == (4, 8)
    assert np.array_equal(q.vertices[:, 0:3], qv[:, 0:3])
    assert np.array_equal(q.vertices[:, 4:7], qv[:, 4:7])
    # u8 normalized uvs: x / 255 in f32
    want_u = (np.round(qv[:, 3] * 255).astype(np.uint8).astype(np.float32) / np.float32(255)).astype(np.float32)
    assert np.array_equal(q.vertices[:, 3], want_u)
    assert np.array_equal(q.triangles, qt) and q.triangles.dtype == np.uint32
    assert np.array_equal(q.bounds, np.array([0, 0, 0, 1, 1, 0], np.float32))
    b = sc.meshes[(1, 0)]
    assert np.array_equal(b.vertices, bv)  # interleaved view, float uvs
    assert np.array_equal(b.triangles, bt)  # the index past the last triple is dropped
    assert np.array_equal(b.bounds[:3], bv[:, 0:3].min(axis=0))
    # scenes and transforms
    assert [s.name for s in sc.scenes] == ["main", "unnamed scene #1"]
    main = sc.scenes[0].instances
    assert [i.mesh_index for i in main] == [(0, 0), (1, 0)]
    t0 = gltf.trs_matrix([1, 2, 3], [0, 0, 0, 1], [2, 2, 2])
    assert np.array_equal(main[0].transform, gltf.mat4_mul(t0, np.asarray(rot_z, np.float32)))
    assert np.array_equal(main[1].transform, np.eye(4, dtype=np.float32).reshape(16))
    # float64 check of the composed matrix: p -> 2 (R p + (5,6,7)) + (1,2,3), R (1,0,0) = (0,-1,0)
    m = main[0].transform.reshape(4, 4).T.astype(np.float64)  # row-major
    p = np.array([1.0, 0.0, 0.0, 1.0])
    assert np.allclose(m @ p, [2 * 5 + 1, 2 * (6 - 1) + 2, 2 * 7 + 3, 1])
    assert "non-uniform scale" in caplog.text
    meshes, scenes = sc.into_meshes_and_scenes()
    assert len(meshes) == 2 and meshes[0] is q and meshes[1] is b
    assert [i.mesh_index for i in scenes[0].instances] == [0, 1]
    ids, tf = gltf.instance_arrays(scenes[1])
    assert ids.tolist() == [1] and tf.shape == (1, 16)


def test_mat4_mul_order_and_trs():
    rng = np.random.default_rng(7)
    a = rng.normal(size=16).astype(np.float32)
    b = rng.normal(size=16).astype(np.float32)
    got = gltf.mat4_mul(a, b).reshape(4, 4).T.astype(np.float64)
    ref = a.reshape(4, 4).T.astype(np.float64) @ b.reshape(4, 4).T.astype(np.float64)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-5)
    # quaternion for 90 degrees about z: x axis -> y axis
    s = np.float32(np.sqrt(0.5))
    r = gltf.trs_matrix([0, 0, 0], [0, 0, s, s], [1, 1, 1]).reshape(4, 4).T.astype(np.float64)
    assert np.allclose(r @ [1, 0, 0, 1], [0, 1, 0, 1], atol=1e-6)


def test_missing_attribute_is_an_error(tmp_path):
    buf = gltf_files.buffer()
    qv, qt = _quad()
    p = gltf_files.mesh_primitive(buf, qv, qt)
    del p["attributes"]["NORMAL"]
    path = gltf_files.write(str(tmp_path / "x"), {"meshes": [{"primitives": [p]}], "nodes": [], "scenes": []},
                            buf, "gltf")
    with pytest.raises(ValueError, match="normals"):
        gltf.GltfScenes.load(path)


def _one_mesh_doc(buf, **prim_kw):
    qv, qt = _quad()
    p = gltf_files.mesh_primitive(buf, qv, qt)
    p.update(prim_kw)
    return {"meshes": [{"primitives": [p]}], "nodes": [{"mesh": 0}], "scenes": [{"nodes": [0]}]}, p


def test_sparse_accessor_is_rejected(tmp_path):
    buf = gltf_files.buffer()
    doc, p = _one_mesh_doc(buf)
    buf.accessors[p["attributes"]["POSITION"]]["sparse"] = {"count": 1}
    path = gltf_files.write(str(tmp_path / "s"), doc, buf, "gltf")
    with pytest.raises(ValueError, match="sparse"):
        gltf.GltfScenes.load(path)


def test_missing_indices_is_an_error(tmp_path):
    buf = gltf_files.buffer()
    doc, p = _one_mesh_doc(buf)
    del p["indices"]
    path = gltf_files.write(str(tmp_path / "i"), doc, buf, "glb")
    with pytest.raises(ValueError, match="indices"):
        gltf.GltfScenes.load(path)


def test_glb_version_and_cycles(tmp_path):
    buf = gltf_files.buffer()
    doc, _ = _one_mesh_doc(buf)
    path = gltf_files.write(str(tmp_path / "v"), doc, buf, "glb")
    data = bytearray(open(path, "rb").read())
    data[4] = 1  # version 1
    bad = str(tmp_path / "v" / "bad.glb")
    open(bad, "wb").write(bytes(data))
    with pytest.raises(ValueError, match="version"):
        gltf.GltfScenes.load(bad)
    buf2 = gltf_files.buffer()
    doc2, _ = _one_mesh_doc(buf2)
    doc2["nodes"] = [{"mesh": 0, "children": [1]}, {"children": [0]}]
    path2 = gltf_files.write(str(tmp_path / "c"), doc2, buf2, "gltf")
    with pytest.raises(ValueError, match="cycle"):
        gltf.GltfScenes.load(path2)


def test_directory_without_gltf(tmp_path):
    (tmp_path / "empty").mkdir()
    with pytest.raises(FileNotFoundError):
        gltf.GltfScenes.load(str(tmp_path / "empty"))
