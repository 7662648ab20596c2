"""Two-level closest-hit traversal, TLAS -> instance -> BLAS (needs a B200).

The scene comes from one batched build (every mesh's BLAS plus the TLAS over
the instances' world boxes), laid out as marigold uploads it for its scene
shader (marigold/assets/shaders/slang/lib/scene.slang:91-220). The traversal
(mgbvh_trace_scene_dev) must find exactly the brute-force hits: same
instance, same triangle and the same distance bit for bit, since both test
each triangle in the instance's mesh space with the same arithmetic. The GPU
brute force is itself checked against the CPU oracle's.
"""
import numpy as np
import pytest

from marigold_b200 import BvhSettings, _lib, build_batch_device, synth
from marigold_b200.bvh import Scene, trace_scene_device

pytestmark = pytest.mark.gpu


def make_scene(seed=5, n_meshes=10, n_inst=60, lo=20, hi=3000, **kw):
    import torch
    meshes, bounds, _ = synth.batched_scene(seed=seed, n_meshes=n_meshes, n_instances=1, lo=lo, hi=hi)
    ids, xf = synth.scene_instances(seed + 1, n_meshes, n_inst)
    # translations shrunk from [-100, 100]^3 to [-3, 3]^3: instances of unit-size
    # meshes crowd together, so most rays meet some of them (and overlap)
    xf = xf.copy()
    xf[:, 12:15] *= np.float32(0.03)
    boxes = synth.instance_aabbs(bounds, ids, xf)
    dmeshes = [(torch.from_numpy(v).cuda(), torch.from_numpy(t.view(np.int32)).cuda()) for v, t in meshes]
    descs = [{"vertices": v, "triangles": t, "bounds": b} for (v, t), b in zip(dmeshes, bounds)]
    descs.append({"aabbs": torch.from_numpy(boxes).cuda()})
    total = sum(t.shape[0] for _, t in meshes) + n_inst
    slots = sum(2 * t.shape[0] - 1 for _, t in meshes) + 2 * n_inst - 1
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(total, dtype=torch.int32, device="cuda")
    ctx = _lib.Context(0)
    offs, rc, _ = build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens, **kw)
    torch.cuda.synchronize()
    ctx.close()
    assert rc >= 0
    multi = kw.get("max_leaf_objects", 1) > 1
    scene = Scene.from_batch(dmeshes, offs, nodes, lens if multi else None, perm,
                             torch.from_numpy(ids.view(np.int32)).cuda(), torch.from_numpy(xf).cuda())
    lo3, hi3 = boxes[:, :3].min(0), boxes[:, 3:].max(0)
    return scene, (lo3, hi3), xf, ids


def compare(a, b):
    ta, ia, pa = (x.cpu().numpy() for x in a[:3])
    tb, ib, pb = (x.cpu().numpy() for x in b[:3])
    bad = (ia != ib) | (pa != pb) | (ta.view(np.uint32) != tb.view(np.uint32))
    return int(bad.sum()), int((pa != -1).sum())


@pytest.mark.parametrize("kw", [{}, {"max_leaf_objects": 4}])
def test_traversal_equals_bruteforce(kw):
    import torch
    scene, (lo, hi), _, _ = make_scene(**kw)
    tr = _lib.Tracer(0)
    scene.bind(tr)
    rays = torch.from_numpy(synth.rays_in_box(4096, lo, hi, seed=3)).cuda()
    got = trace_scene_device(tr, rays)
    want = trace_scene_device(tr, rays, bruteforce=True)
    culled = trace_scene_device(tr, rays, bruteforce=True, cull=True)
    mism, hits = compare(got, want)
    assert hits > 500, hits
    assert mism == 0, (mism, hits)
    assert compare(culled, want)[0] == 0
    nodes, boxes, tris = got[3]
    assert nodes > 0 and boxes > 0 and tris > 0
    tr.close()


def test_gpu_bruteforce_equals_cpu_oracle(oracle):
    import torch
    scene, (lo, hi), _, _ = make_scene(seed=8, n_meshes=6, n_inst=25, hi=1500)
    tr = _lib.Tracer(0)
    scene.bind(tr)
    r = synth.rays_in_box(256, lo, hi, seed=4)
    g = trace_scene_device(tr, torch.from_numpy(r).cuda(), bruteforce=True)
    o = oracle.trace_scene_bruteforce(scene.vertices.cpu().numpy(), scene.triangles.cpu().numpy().view(np.uint32),
                                      scene.meshes.cpu().numpy(), scene.instances.cpu().numpy(), r)
    gt, gi, gp = (x.cpu().numpy() for x in g[:3])
    assert np.array_equal(gt.view(np.uint32), o[0].view(np.uint32))
    assert np.array_equal(gi.view(np.uint32), o[1]) and np.array_equal(gp.view(np.uint32), o[2])
    assert (o[2] != 0xFFFFFFFF).sum() > 20
    tr.close()


def test_distances_are_world_units():
    """t is the world ray's parameter in every instance, scaled ones
    included: the hit point o + t d lies on the hit triangle's plane in world
    space (float64 check, relative 1e-4 of the scene size)."""
    import torch
    scene, (lo, hi), xf, ids = make_scene(seed=11, n_meshes=5, n_inst=30, hi=2000)
    tr = _lib.Tracer(0)
    scene.bind(tr)
    r = synth.rays_in_box(2048, lo, hi, seed=5)
    t, inst, tri, _, _ = trace_scene_device(tr, torch.from_numpy(r).cuda())
    t, inst, tri = t.cpu().numpy(), inst.cpu().numpy(), tri.cpu().numpy()
    order = scene.instance_order.cpu().numpy()  # TLAS slot -> original instance
    verts = scene.vertices.cpu().numpy().astype(np.float64)
    tris = scene.triangles.cpu().numpy().astype(np.int64)
    mtab = scene.meshes.cpu().numpy().view(np.uint32)
    scale = float(np.abs(hi - lo).max())
    checked = 0
    for k in np.nonzero(tri != -1)[0][:400]:
        orig = order[inst[k]]
        mesh = ids[orig]
        vo = int(mtab[mesh, 3])
        a, b, c = (verts[vo + tris[tri[k], q]] for q in range(3))
        m = xf[orig].astype(np.float64).reshape(4, 4).T  # mesh -> world, row-major math matrix
        w = [m[:3, :3] @ p + m[:3, 3] for p in (a, b, c)]
        n = np.cross(w[1] - w[0], w[2] - w[0])
        p = r[k, 0:3].astype(np.float64) + t[k] * r[k, 4:7].astype(np.float64)
        assert abs(np.dot(n / np.linalg.norm(n), p - w[0])) < 1e-4 * scale, k
        checked += 1
    assert checked > 100
    tr.close()
