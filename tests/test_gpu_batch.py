"""Batched builds (many BLAS + the TLAS in one pass) vs one build per mesh.

Every mesh of a batch must come out exactly as building it alone: the same
node words, lengths and permutation. Single builds are themselves checked
against the oracle (test_gpu_parity); a few meshes here are also compared
with the oracle directly. The switch-over between level passes and subtree
kernels is a speed knob and must not change any tree.
"""
import numpy as np
import pytest

from marigold_b200 import BvhSettings, _lib, build_batch_device, synth
from tests.gpuhelp import gpu_build
from tests.treecheck import compare_exact

pytestmark = pytest.mark.gpu


def scene(n_meshes=40, n_inst=300, lo=1, hi=20000, seed=7):
    meshes, bounds, inst = synth.batched_scene(seed=seed, n_meshes=n_meshes, n_instances=n_inst,
                                               lo=lo, hi=hi)
    # edge cases: an empty mesh and a one-triangle mesh
    v1, t1 = synth.random_triangles(1, seed=99)
    meshes = meshes + [(np.zeros((0, 8), np.float32), np.zeros((0, 3), np.uint32)), (v1, t1)]
    bounds = np.concatenate([bounds, np.zeros((1, 6), np.float32), synth.mesh_bounds(v1)[None]])
    return meshes, bounds, inst


def run_batch(meshes, bounds, inst, medium_max=None, **kw):
    import torch
    ctx = _lib.Context(0)
    if medium_max:
        ctx.check(ctx.L.mgbvh_set_tuning(ctx.ptr, medium_max))
    descs = []
    for (v, t), b in zip(meshes, bounds):
        descs.append({"vertices": torch.from_numpy(v).cuda(),
                      "triangles": torch.from_numpy(t.view(np.int32)).cuda(),
                      "bounds": b if t.shape[0] else None})
    descs.append({"aabbs": torch.from_numpy(inst).cuda()})  # the TLAS: bounds None
    total = sum(t.shape[0] for _, t in meshes) + inst.shape[0]
    slots = sum(2 * t.shape[0] - 1 for _, t in meshes if t.shape[0]) + 2 * inst.shape[0] - 1
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(total, dtype=torch.int32, device="cuda")
    offs, rc, st = build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens, **kw)
    torch.cuda.synchronize()
    ctx.close()
    return (offs, rc, nodes.cpu().numpy().view(np.uint32).reshape(-1, 8),
            lens.cpu().numpy().view(np.uint32), perm.cpu().numpy().view(np.uint32))


def check_against_single(meshes, bounds, inst, res, **kw):
    offs, rc, nodes, lens, perm = res
    assert rc >= 0
    ctx = _lib.Context(0)
    first = 0
    single_kw = dict(kw)
    if "min_leaf_objects" in single_kw:
        single_kw["min_leaf"] = single_kw.pop("min_leaf_objects")
    if "max_leaf_objects" in single_kw:
        single_kw["max_leaf"] = single_kw.pop("max_leaf_objects")
    objs = [("mesh", v, t, b) for (v, t), b in zip(meshes, bounds)] + [("tlas", None, inst, None)]
    for m, (kind, v, t, b) in enumerate(objs):
        n = t.shape[0]
        if kind == "tlas":
            g = gpu_build(ctx, aabbs=inst, **single_kw)
        elif n == 0:
            assert offs[m + 1] == offs[m]
            continue
        else:
            g = gpu_build(ctx, vertices=v, triangles=t, root_bounds=b, **single_kw)
        got_nodes = nodes[offs[m]:offs[m + 1]]
        got_lens = lens[offs[m]:offs[m + 1]]
        got_perm = perm[first:first + n]
        msg = compare_exact(got_nodes, got_lens, got_perm, g["nodes"], g["lens"], g["perm"])
        assert msg is None, f"mesh {m} ({kind}, {n} objects): {msg}"
        first += n
    ctx.close()


def test_batch_equals_single_builds():
    meshes, bounds, inst = scene()
    check_against_single(meshes, bounds, inst, run_batch(meshes, bounds, inst))


def test_batch_multi_object_leaves_compaction():
    meshes, bounds, inst = scene(n_meshes=12, n_inst=100, hi=5000, seed=8)
    kw = dict(min_leaf_objects=2, max_leaf_objects=4)
    check_against_single(meshes, bounds, inst, run_batch(meshes, bounds, inst, **kw), **kw)


def test_switch_over_does_not_change_trees():
    meshes, bounds, inst = scene(n_meshes=16, n_inst=64, hi=50000, seed=9)
    a = run_batch(meshes, bounds, inst)
    b = run_batch(meshes, bounds, inst, medium_max=64)
    assert a[0] == b[0]
    msg = compare_exact(a[2], a[3], a[4], b[2], b[3], b[4])
    assert msg is None, msg


def test_batch_meshes_match_oracle():
    from oracle import oracle as orc
    meshes, bounds, inst = scene(n_meshes=6, n_inst=50, hi=3000, seed=10)
    offs, rc, nodes, lens, perm = run_batch(meshes, bounds, inst)
    first = 0
    for m, ((v, t), b) in enumerate(zip(meshes, bounds)):
        n = t.shape[0]
        if n == 0:
            continue
        o = orc.build(v, t, root_bounds=b)
        msg = compare_exact(nodes[offs[m]:offs[m + 1]], lens[offs[m]:offs[m + 1]],
                            perm[first:first + n], o["nodes"], o["lens"], o["perm"])
        assert msg is None, f"mesh {m}: {msg}"
        first += n
    o = orc.build(aabbs=inst)
    k = len(meshes)
    msg = compare_exact(nodes[offs[k]:offs[k + 1]], lens[offs[k]:offs[k + 1]],
                        perm[first:first + inst.shape[0]], o["nodes"], o["lens"], o["perm"])
    assert msg is None, f"tlas: {msg}"


def test_graph_replay_equals_eager_build():
    import torch
    meshes, bounds, inst = scene(n_meshes=24, n_inst=200, hi=60000, seed=12)
    ctx = _lib.Context(0)
    ctx.check(ctx.L.mgbvh_set_graph_capture(ctx.ptr, 1))
    stream = torch.cuda.Stream()  # capture needs a stream other than the legacy default
    descs = [{"vertices": torch.from_numpy(v).cuda(), "triangles": torch.from_numpy(t.view(np.int32)).cuda(),
              "bounds": b if t.shape[0] else None} for (v, t), b in zip(meshes, bounds)]
    descs.append({"aabbs": torch.from_numpy(inst).cuda()})
    total = sum(t.shape[0] for _, t in meshes) + inst.shape[0]
    slots = sum(2 * t.shape[0] - 1 for _, t in meshes if t.shape[0]) + 2 * inst.shape[0] - 1
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(total, dtype=torch.int32, device="cuda")
    results = []
    for k in range(3):
        nodes.zero_()
        perm.zero_()
        torch.cuda.synchronize()
        offs, rc, st = build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens,
                                          stream=stream)
        stream.synchronize()
        results.append((offs, st["graph_replay"], nodes.cpu().numpy().copy(),
                        lens.cpu().numpy().copy(), perm.cpu().numpy().copy()))
    assert results[0][1] == 0 and results[1][1] == 1 and results[2][1] == 1
    for r in results[1:]:
        assert r[0] == results[0][0]
        msg = compare_exact(r[2].view(np.uint32).reshape(-1, 8), r[3], r[4],
                            results[0][2].view(np.uint32).reshape(-1, 8), results[0][3], results[0][4])
        assert msg is None, msg
    ctx.close()
