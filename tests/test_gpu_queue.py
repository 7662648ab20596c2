"""The persistent batched build (mgbvh_set_batch_mode MGBVH_BATCH_QUEUE;
needs a B200).

One launch takes node tasks of every mesh and the TLAS from device-side
queues. It must give exactly the trees of the level-pass batched build (which
tests/test_gpu_batch.py checks against single builds and the oracle): the
same node words, lengths and permutations, for both leaf-size profiles, both
subtree-CTA sizes, the knob profiles, forced medians, and graph replay. Its
waits are bounded: a build whose queue holds a task that never arrives ends
with MGBVH_ERR_TIMEOUT and leaves the context usable.
"""
import numpy as np
import pytest

from marigold_b200 import BvhSettings, MgbvhError, _lib, build_batch_device, synth
from tests import median_cases as mc
from tests.treecheck import compare_exact

pytestmark = pytest.mark.gpu


def scene(seed=7, n_meshes=30, n_inst=300, lo=1, hi=30000, extra=()):
    import torch
    meshes, bounds, inst = synth.batched_scene(seed=seed, n_meshes=n_meshes, n_instances=n_inst, lo=lo, hi=hi)
    descs = [{"vertices": torch.from_numpy(v).cuda(), "triangles": torch.from_numpy(t.view(np.int32)).cuda(),
              "bounds": b} for (v, t), b in zip(meshes, bounds)]
    counts = [t.shape[0] for _, t in meshes]
    for boxes in extra:  # AABB lists (forced-median inputs and the like)
        descs.append({"aabbs": torch.from_numpy(boxes).cuda()})
        counts.append(boxes.shape[0])
    descs.append({"aabbs": torch.from_numpy(inst).cuda()})  # the TLAS
    counts.append(inst.shape[0])
    return descs, counts


def run(descs, counts, queue, medium_max=None, graph=False, reps=1, settings=None, **kw):
    import torch
    ctx = _lib.Context(0)
    ctx.set_batch_mode(queue)
    if medium_max:
        ctx.set_tuning(medium_max)
    if graph:
        ctx.set_graph_capture(True)
    slots = sum(2 * n - 1 for n in counts if n)
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(sum(counts), dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    out = []
    for _ in range(reps):
        nodes.zero_()
        perm.zero_()
        torch.cuda.synchronize()
        offs, rc, st = build_batch_device(ctx, settings or BvhSettings(), descs, nodes, perm, out_lens=lens,
                                          stream=stream, **kw)
        stream.synchronize()
        assert rc >= 0
        out.append((offs, st, nodes.cpu().numpy().view(np.uint32).reshape(-1, 8).copy(),
                    lens.cpu().numpy().view(np.uint32).copy(), perm.cpu().numpy().view(np.uint32).copy()))
    ctx.close()
    return out


def same(a, b):
    assert a[0] == b[0]
    n = a[0][-1]
    msg = compare_exact(a[2][:n], a[3][:n], a[4], b[2][:n], b[3][:n], b[4])
    assert msg is None, msg


@pytest.mark.parametrize("medium_max", [1024, 512, 64])
@pytest.mark.parametrize("leaf", [dict(), dict(min_leaf_objects=2, max_leaf_objects=4)])
def test_queue_equals_level_passes(medium_max, leaf):
    descs, counts = scene()
    a = run(descs, counts, False, medium_max, **leaf)[0]
    b = run(descs, counts, True, medium_max, **leaf)[0]
    same(a, b)
    assert b[1]["kernel_launches"] <= 6  # prep, roots, the persistent launch


@pytest.mark.parametrize("knobs", [dict(bins=16, adaptive_max_n=0), dict(adaptive_steps=16), dict(max_depth=9)])
def test_queue_knob_profiles(knobs):
    descs, counts = scene(seed=9, n_meshes=16, hi=20000)
    s = BvhSettings(**knobs)
    same(run(descs, counts, False, settings=s)[0], run(descs, counts, True, settings=s)[0])


def test_queue_with_forced_medians(oracle):
    extra = (mc.coincident_boxes(5000, 3), mc.cluster_in_mesh(8000, 2000, 4), mc.outlier_boxes(3000, 5))
    descs, counts = scene(seed=11, n_meshes=8, hi=10000, extra=extra)
    a = run(descs, counts, False)[0]
    b = run(descs, counts, True)[0]
    same(a, b)
    # and the coincident list against the oracle directly
    m = 8
    o = oracle.build(aabbs=extra[0])
    first = sum(counts[:m])
    offs = b[0]
    msg = compare_exact(b[2][offs[m]:offs[m + 1]], b[3][offs[m]:offs[m + 1]], b[4][first:first + counts[m]],
                        o["nodes"], o["lens"], o["perm"])
    assert msg is None, msg


def test_queue_graph_replay():
    descs, counts = scene(seed=12, n_meshes=24, hi=60000)
    res = run(descs, counts, True, graph=True, reps=3)
    assert [r[1]["graph_replay"] for r in res] == [0, 1, 1]
    for r in res[1:]:
        same(r, res[0])
    same(res[0], run(descs, counts, False)[0])


def test_queue_wait_runs_out_and_context_stays_usable():
    """A task counted as pending that never arrives: every CTA's wait runs
    out after the limit (0.2 s here), the launch ends, the build returns
    MGBVH_ERR_TIMEOUT; the next build on the context is correct."""
    import time
    import torch
    descs, counts = scene(seed=13, n_meshes=6, hi=5000)
    want = run(descs, counts, False)[0]
    ctx = _lib.Context(0)
    ctx.set_batch_mode(True)
    ctx.set_queue_limits(200000, 1)
    slots = sum(2 * n - 1 for n in counts if n)
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(sum(counts), dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    with pytest.raises(MgbvhError) as e:
        build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens)
    assert e.value.status == _lib.ERR_TIMEOUT
    assert time.perf_counter() - t0 < 30
    assert "ran out" in ctx.last_error()
    ctx.set_queue_limits(0, 0)
    offs, rc, st = build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens)
    torch.cuda.synchronize()
    got = (offs, st, nodes.cpu().numpy().view(np.uint32).reshape(-1, 8), lens.cpu().numpy().view(np.uint32),
           perm.cpu().numpy().view(np.uint32))
    same(got, want)
    ctx.close()
