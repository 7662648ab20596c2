"""GPU instance AABBs (the TLAS input of marigold's scene upload,
marigold/src/app/data/scene/model.rs:191-234) against the oracle, bit for
bit, and a batched scene build fed from them."""
from __future__ import annotations

import numpy as np
import pytest

from marigold_b200 import BvhSettings, _lib, build_batch_device, synth
from marigold_b200.bvh import instance_aabbs_device

from tests.treecheck import compare_exact

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,m", [(1, 1), (4096, 512), (100000, 37)])
def test_instance_aabbs_match_oracle(oracle, gpu_ctx, n, m):
    rng = np.random.default_rng(n + m)
    bounds = np.sort(rng.normal(size=(m, 2, 3)).astype(np.float32), axis=1).reshape(m, 6)
    bounds[0, [0, 3]] = [-0.0, 0.0]
    ids = rng.integers(0, m, n).astype(np.uint32)
    xf = rng.normal(size=(n, 16)).astype(np.float32)
    xf[:, [3, 7, 11]] = 0.0
    xf[:, 15] = 1.0
    xf[: n // 3, 1] = 0.0
    out = torch.empty((n, 6), dtype=torch.float32, device="cuda")
    instance_aabbs_device(gpu_ctx, _dev(bounds), _dev(ids.view(np.int32)), _dev(xf), out)
    want, bad = oracle.instance_aabbs(bounds, ids, xf)
    assert bad == 0
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_instance_aabbs_bad_index(gpu_ctx):
    bounds = np.zeros((2, 6), np.float32)
    ids = np.array([0, 2, 1], np.uint32)
    xf = np.tile(np.eye(4, dtype=np.float32).T.reshape(16), (3, 1))
    out = torch.empty((3, 6), dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.MgbvhError) as e:
        instance_aabbs_device(gpu_ctx, _dev(bounds), _dev(ids.view(np.int32)), _dev(xf), out)
    assert e.value.status == _lib.ERR_INVALID_ARG
    # the context stays usable
    instance_aabbs_device(gpu_ctx, _dev(bounds), _dev(ids[:1].view(np.int32)), _dev(xf[:1]), out[:1])


def test_batched_scene_from_gpu_instances(gpu_ctx):
    """The TLAS of a batched build fed by the GPU instance boxes equals the
    one built from the host restatement's boxes (the same floats)."""
    meshes, bounds, inst = synth.batched_scene(seed=5, n_meshes=12, n_instances=2000, lo=50, hi=5000)
    ids, xf = synth.scene_instances(5, 12, 2000)
    d_inst = torch.empty((2000, 6), dtype=torch.float32, device="cuda")
    instance_aabbs_device(gpu_ctx, _dev(bounds), _dev(ids.view(np.int32)), _dev(xf), d_inst)
    assert np.array_equal(d_inst.cpu().numpy().view(np.uint32), inst.view(np.uint32))
    results = []
    for tlas in (d_inst, _dev(inst)):
        descs = [{"vertices": _dev(v), "triangles": _dev(t.view(np.int32)), "bounds": b}
                 for (v, t), b in zip(meshes, bounds)]
        descs.append({"aabbs": tlas})
        total = sum(t.shape[0] for _, t in meshes) + 2000
        slots = sum(2 * t.shape[0] - 1 for _, t in meshes) + 2 * 2000 - 1
        nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
        lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
        perm = torch.zeros(total, dtype=torch.int32, device="cuda")
        offs, rc, _ = build_batch_device(gpu_ctx, BvhSettings(), descs, nodes, perm, out_lens=lens)
        torch.cuda.synchronize()
        assert rc >= 0
        results.append((nodes.cpu().numpy().view(np.uint32).reshape(-1, 8), lens.cpu().numpy(),
                        perm.cpu().numpy()))
    assert compare_exact(*results[0], *results[1]) is None
