"""A glTF scene from file to trees on the GPU (needs a B200): the loader's
meshes go to device buffers, every BLAS builds in one batched pass with the
accessor bounds as root bounds, and the TLAS over the scene's instance boxes
(computed on the GPU from the instance transforms) in the same pass. Each
tree equals the oracle's, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from marigold_b200 import BvhSettings, build_batch_device, gltf, synth
from marigold_b200.bvh import instance_aabbs_device
from tests import gltf_files
from tests.treecheck import compare_exact

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_gltf_scene_to_trees(tmp_path, oracle, gpu_ctx):
    buf = gltf_files.buffer()
    prims = []
    for k, n in enumerate((3000, 40000, 17)):
        v, t = synth.random_triangles(n, seed=700 + k)
        prims.append(gltf_files.mesh_primitive(buf, v, t, interleaved=(k == 1),
                                               index_type=5125 if n > 20000 else 5123))
    xf = [[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 10, 0, 0, 1], [0, 1, 0, 0, -1, 0, 0, 0, 0, 0, 1, 0, 0, 5, 0, 1]]
    doc = {"meshes": [{"primitives": prims[:2]}, {"primitives": [prims[2]]}],
           "nodes": [{"matrix": xf[0], "mesh": 0, "children": [1, 2]},
                     {"matrix": xf[1], "mesh": 1},
                     {"translation": [0, 0, 3], "rotation": [0, 0.6, 0, 0.8], "scale": [2, 2, 2], "mesh": 0}],
           "scenes": [{"name": "s", "nodes": [0]}]}
    path = gltf_files.write(str(tmp_path / "scene"), doc, buf, "glb")
    meshes, scenes = gltf.GltfScenes.load(path).into_meshes_and_scenes()
    assert [m.triangles.shape[0] for m in meshes] == [3000, 40000, 17]
    ids, tfs = gltf.instance_arrays(scenes[0])
    assert ids.tolist() == [0, 1, 2, 0, 1]  # node 0: both primitives of mesh 0, node 1: mesh 1, node 2: mesh 0

    bounds = np.stack([m.bounds for m in meshes])
    d_inst = torch.empty((ids.shape[0], 6), dtype=torch.float32, device="cuda")
    instance_aabbs_device(gpu_ctx, torch.from_numpy(bounds).cuda(), torch.from_numpy(ids.view(np.int32)).cuda(),
                          torch.from_numpy(tfs).cuda(), d_inst)
    inst = synth.instance_aabbs(bounds, ids, tfs)
    assert np.array_equal(d_inst.cpu().numpy().view(np.uint32), inst.view(np.uint32))

    descs = gltf.to_device(meshes) + [{"aabbs": d_inst}]
    total = sum(m.triangles.shape[0] for m in meshes) + ids.shape[0]
    slots = sum(2 * m.triangles.shape[0] - 1 for m in meshes) + 2 * ids.shape[0] - 1
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(total, dtype=torch.int32, device="cuda")
    offs, rc, _ = build_batch_device(gpu_ctx, BvhSettings(), descs, nodes, perm, out_lens=lens)
    torch.cuda.synchronize()
    assert rc >= 0
    nodes = nodes.cpu().numpy().view(np.uint32).reshape(-1, 8)
    lens = lens.cpu().numpy().view(np.uint32)
    perm = perm.cpu().numpy().view(np.uint32)
    first = 0
    for m, mesh in enumerate(meshes + [None]):
        if mesh is None:
            o = oracle.build(aabbs=inst)
            n = inst.shape[0]
        else:
            o = oracle.build(mesh.vertices, mesh.triangles, root_bounds=mesh.bounds)
            n = mesh.triangles.shape[0]
        msg = compare_exact(nodes[offs[m]:offs[m + 1]], lens[offs[m]:offs[m + 1]], perm[first:first + n],
                            o["nodes"], o["lens"], o["perm"])
        assert msg is None, f"tree {m}: {msg}"
        first += n
