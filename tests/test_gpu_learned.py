"""GPU checks of the learned split proposer.

* the training kernels (forward, backward, Adam) against the float64 CPU
  reference of the network, on the BF16 weights the kernels use;
* the builder's training samples (features, full-sweep labels, gain flags,
  both costs) against the oracle's samples of the same plain build, node by
  node (matched by start and object count);
* builds with a network in the loop: with fixed proposals, word for word
  the oracle's restatement of the learned split rule; with any network,
  valid trees (the reference's invariants); with the trained network, SAH
  cost below plain binned and within 1% of the full sweep, and a gain over
  an untrained network.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from marigold_b200 import _lib, learned, synth
from marigold_b200.bvh import NODE_DTYPE, sah_cost

from tests.gpuhelp import gpu_build
from tests.treecheck import check_tree, compare_exact

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def mlp_ref():
    from oracle import mlp_ref as m
    return m


def _bf16_float(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32)


def _batch(B, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(scale=0.6, size=(B, 24)).astype(np.float32)
    label = rng.integers(0, 48, B).astype(np.uint32)
    label[::7] = 0xFFFFFFFF
    gain = (rng.random(B) < 0.3).astype(np.float32)
    return x, label, gain


@pytest.mark.parametrize("B", [1, 100, 1000])
def test_train_step_gradient_matches_oracle(mlp_ref, B):
    L = _lib.load()
    bits = learned.to_bf16_bits(learned.init_params(11))
    x, label, gain = _batch(B, 40 + B)
    w = torch.from_numpy(bits.view(np.int16)).cuda()
    dx, dl, dg = (torch.from_numpy(a).cuda() for a in (x, label.view(np.int32), gain))
    grad = torch.zeros(learned.NPARAM, dtype=torch.float32, device="cuda")
    loss = torch.zeros(2, dtype=torch.float32, device="cuda")
    assert L.mgbvh_mlp_train_step_dev(_vp(dx), _vp(dl), _vp(dg), B, _vp(w), _vp(grad), _vp(loss),
                                      None) == 0
    torch.cuda.synchronize()
    ref_loss, ref_g = mlp_ref.loss_and_grad(_bf16_float(bits), x, label, gain)
    g = grad.cpu().numpy().astype(np.float64)
    scale = np.abs(ref_g).max()
    err = np.abs(g - ref_g).max()
    assert err <= 2e-5 * scale + 1e-8, (err, scale)
    # every parameter block receives its gradient
    for s, e in ((0, 1536), (1536, 1600), (1600, 5696), (5696, 5760), (5760, 8896), (8896, 8945)):
        assert np.abs(g[s:e]).max() > 0
    lsum = float(loss.sum().item()) / B
    assert abs(lsum - ref_loss) <= 1e-5 * abs(ref_loss) + 1e-6


def test_forward_matches_oracle(mlp_ref):
    L = _lib.load()
    bits = learned.to_bf16_bits(learned.init_params(12))
    x, _, _ = _batch(333, 9)
    w = torch.from_numpy(bits.view(np.int16)).cuda()
    dx = torch.from_numpy(x).cuda()
    out = torch.empty(333 * 49, dtype=torch.float32, device="cuda")
    assert L.mgbvh_mlp_forward_dev(_vp(dx), 333, _vp(w), _vp(out), None) == 0
    ref, _ = mlp_ref.forward(_bf16_float(bits), x)
    got = out.view(333, 49).cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def test_adam_step():
    L = _lib.load()
    rng = np.random.default_rng(4)
    p = learned.init_params(13)
    g = rng.normal(scale=1e-2, size=learned.NPARAM).astype(np.float32)
    m0 = rng.normal(scale=1e-3, size=learned.NPARAM).astype(np.float32)
    v0 = np.abs(rng.normal(scale=1e-5, size=learned.NPARAM)).astype(np.float32)
    master, grad, m, v = (torch.from_numpy(a.copy()).cuda() for a in (p, g, m0, v0))
    w = torch.zeros(learned.NPARAM, dtype=torch.int16, device="cuda")
    step, lr, b1, b2, eps = 3, 1e-3, 0.9, 0.999, 1e-8
    assert L.mgbvh_mlp_adam_dev(_vp(master), _vp(w), _vp(grad), _vp(m), _vp(v), step, lr, b1, b2,
                                eps, None) == 0
    torch.cuda.synchronize()
    mr = b1 * m0.astype(np.float64) + (1 - b1) * g
    vr = b2 * v0.astype(np.float64) + (1 - b2) * g.astype(np.float64) ** 2
    pr = p - lr * (mr / (1 - b1 ** step)) / (np.sqrt(vr / (1 - b2 ** step)) + eps)
    got = master.cpu().numpy()
    assert np.abs(got - pr).max() <= 1e-6
    assert np.array_equal(w.cpu().numpy().view(np.uint16), learned.to_bf16_bits(got))


@pytest.fixture()
def fresh_ctx():
    ctx = _lib.Context(0)
    ctx.set_tuning(1024)
    yield ctx
    ctx.close()


@pytest.mark.parametrize("mesh", ["random", "icosphere"])
def test_samples_match_oracle(oracle, fresh_ctx, mesh):
    """Every binned node of 33..8192 objects (subtree kernel up to 1024, level
    passes above) yields one sample, equal to the oracle's sample of the same
    node: features to FP32 rounding, label, gain and both costs exactly."""
    if mesh == "random":
        v, t = synth.random_triangles(20000, seed=77)
    else:
        v, t = synth.noisy_icosphere(5, seed=78)
    cap = t.shape[0]
    out = torch.zeros(cap * learned.SAMPLE_WIDTH, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    fresh_ctx.set_sample_output(out, cap, cnt)
    r = gpu_build(fresh_ctx, v, t)
    assert r["status"] == 0, r["error"]
    fresh_ctx.set_sample_output(None)
    k = int(cnt.item())
    assert 0 < k <= cap
    gs = out[: k * 30].view(k, 30).cpu().numpy()
    os_ = oracle.sample_nodes(v, t, min_n=33)
    # the plain tree is the reference's: sampling must not change it
    ref = oracle.build(v, t)
    assert np.array_equal(r["nodes"], ref["nodes"]) and np.array_equal(r["perm"], ref["perm"])
    want = os_[(os_[:, 26] <= 8192) & np.isfinite(os_[:, 27])]
    assert (want[:, 26] > 1024).any()
    key = lambda s: (s[:, 29].astype(np.int64) << 32) | s[:, 26].astype(np.int64)  # noqa: E731
    gk, ok_ = key(gs), key(want)
    assert len(np.unique(gk)) == k
    assert np.array_equal(np.sort(gk), np.sort(ok_))
    gs = gs[np.argsort(gk)]
    want = want[np.argsort(ok_)]
    assert np.abs(gs[:, :24] - want[:, :24]).max() <= 2e-6
    assert np.array_equal(gs[:, 24].view(np.uint32), want[:, 24].view(np.uint32))
    assert np.array_equal(gs[:, 25], want[:, 25])
    assert np.array_equal(gs[:, 27].view(np.uint32), want[:, 27].view(np.uint32))
    assert np.array_equal(gs[:, 28].view(np.uint32), want[:, 28].view(np.uint32))
    assert 0 < gs[:, 25].sum() < k  # some nodes gain from the exact sweep, some do not


def _sah(r):
    return sah_cost(r["nodes"].view(NODE_DTYPE).reshape(-1), r["lens"])


def _learned_build(ctx, v, t, bits, gate):
    w = torch.from_numpy(np.ascontiguousarray(bits).view(np.int16)).cuda()
    ctx.set_split_proposer(w, gate)
    try:
        return gpu_build(ctx, v, t)
    finally:
        ctx.set_split_proposer(None)


def fixed_proposals(p0, p1, refine=1.0):
    """BF16 parameters whose outputs ignore the features: every hidden unit is
    GELU(0) = 0, so the logits are b3 and the two proposals are p0 and p1."""
    p = np.zeros(learned.NPARAM, np.float32)
    p[8896 + p0] = 2.0
    p[8896 + p1] = 1.0
    p[8896 + 48] = refine
    return learned.to_bf16_bits(p)


@pytest.mark.parametrize("mesh,p0,p1,medium_max", [
    ("random", 7, 23, 1024), ("random", 40, 41, 1024), ("random", 8, 24, 512),
    ("icosphere", 39, 7, 1024), ("icosphere", 20, 5, 256), ("random", 15, 31, 1024)])
def test_learned_form_matches_oracle(oracle, fresh_ctx, mesh, p0, p1, medium_max):
    """With fixed proposals the learned form is a deterministic split rule at
    every binned node of 33 or more objects (level passes and subtree kernels
    alike, so the switch-over between them does not change the tree); the
    GPU tree equals the oracle's restatement of it word for word."""
    if mesh == "random":
        v, t = synth.random_triangles(30000, seed=91)
    else:
        v, t = synth.noisy_icosphere(5, seed=93)
    fresh_ctx.set_tuning(medium_max)
    r = _learned_build(fresh_ctx, v, t, fixed_proposals(p0, p1), False)
    assert r["status"] == 0, r["error"]
    ref = oracle.build(v, t, learned=(0xFFFFFFFF, p0, p1))
    assert ref["status"] == 0
    msg = compare_exact(r["nodes"], r["lens"], r["perm"], ref["nodes"], ref["lens"], ref["perm"])
    assert msg is None, msg
    assert r["stats"]["learned_splits"] == ref["stats"]["learned_splits"]
    if (p0, p1) != (15, 31):
        assert ref["stats"]["learned_splits"] > 0
    check_tree(r["nodes"], r["lens"], r["perm"], synth.triangle_aabbs(v, t))


def test_learned_gate(oracle, fresh_ctx):
    """A negative refine logit with the gate on leaves the plain tree; with
    the gate off the proposals are scored anyway."""
    v, t = synth.random_triangles(30000, seed=94)
    plain = gpu_build(fresh_ctx, v, t)
    bits = fixed_proposals(7, 23, refine=-1.0)
    gated = _learned_build(fresh_ctx, v, t, bits, True)
    assert gated["stats"]["learned_splits"] == 0
    assert compare_exact(gated["nodes"], gated["lens"], gated["perm"], plain["nodes"],
                         plain["lens"], plain["perm"]) is None
    ungated = _learned_build(fresh_ctx, v, t, bits, False)
    assert ungated["stats"]["learned_splits"] > 0
    # a plain build right after is the reference's tree again
    again = gpu_build(fresh_ctx, v, t)
    assert np.array_equal(again["nodes"], plain["nodes"])
    assert again["stats"]["learned_splits"] == 0


def test_learned_batch_matches_oracle(oracle):
    """A batched build (many BLAS + the TLAS in one pass) with fixed
    proposals: every tree equals the oracle's learned-form tree."""
    from marigold_b200 import BvhSettings, build_batch_device
    from tests.test_gpu_batch import scene
    meshes, bounds, inst = scene(n_meshes=10, n_inst=3000, lo=1, hi=40000, seed=17)
    ctx = _lib.Context(0)
    p0, p1 = 7, 23
    w = torch.from_numpy(fixed_proposals(p0, p1).view(np.int16)).cuda()
    ctx.set_split_proposer(w, False)
    descs = [{"vertices": torch.from_numpy(v).cuda(), "triangles": torch.from_numpy(t.view(np.int32)).cuda(),
              "bounds": b if t.shape[0] else None} for (v, t), b in zip(meshes, bounds)]
    descs.append({"aabbs": torch.from_numpy(inst).cuda()})
    total = sum(t.shape[0] for _, t in meshes) + inst.shape[0]
    slots = sum(2 * t.shape[0] - 1 for _, t in meshes if t.shape[0]) + 2 * inst.shape[0] - 1
    nodes = torch.zeros(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(slots, dtype=torch.int32, device="cuda")
    perm = torch.zeros(total, dtype=torch.int32, device="cuda")
    offs, rc, st = build_batch_device(ctx, BvhSettings(), descs, nodes, perm, out_lens=lens)
    torch.cuda.synchronize()
    ctx.close()
    assert rc >= 0 and st["learned_splits"] > 0
    nodes = nodes.cpu().numpy().view(np.uint32).reshape(-1, 8)
    lens = lens.cpu().numpy().view(np.uint32)
    perm = perm.cpu().numpy().view(np.uint32)
    first = 0
    objs = [(v, t, b) for (v, t), b in zip(meshes, bounds)] + [(None, inst, None)]
    for m, (v, t, b) in enumerate(objs):
        n = t.shape[0]
        if n == 0:
            continue
        if v is None:
            ref = oracle.build(aabbs=inst, learned=(0xFFFFFFFF, p0, p1))
        else:
            ref = oracle.build(v, t, root_bounds=b, learned=(0xFFFFFFFF, p0, p1))
        msg = compare_exact(nodes[offs[m]:offs[m + 1]], lens[offs[m]:offs[m + 1]], perm[first:first + n],
                            ref["nodes"], ref["lens"], ref["perm"])
        assert msg is None, f"tree {m} ({n} objects): {msg}"
        first += n


@pytest.mark.parametrize("gate", [False, True])
def test_learned_build_valid(fresh_ctx, gate):
    v, t = synth.random_triangles(30000, seed=91)
    r = _learned_build(fresh_ctx, v, t, learned.to_bf16_bits(learned.init_params(5)), gate)
    assert r["status"] == 0, r["error"]
    check_tree(r["nodes"], r["lens"], r["perm"], synth.triangle_aabbs(v, t))


def test_learned_build_deterministic(fresh_ctx):
    v, t = synth.noisy_icosphere(5, seed=92)
    bits = learned.to_bf16_bits(learned.init_params(6))
    a = _learned_build(fresh_ctx, v, t, bits, False)
    b = _learned_build(fresh_ctx, v, t, bits, False)
    assert np.array_equal(a["nodes"], b["nodes"]) and np.array_equal(a["perm"], b["perm"])


def test_trained_network_gains(oracle, fresh_ctx):
    """The committed trained network, on held-out seeds: below plain binned
    SAH, within 1% of the full sweep, and, scoring the same number of
    proposals per node (gate off), more SAH gained than an untrained
    network's proposals give."""
    trained = learned.load_weights()
    untrained = learned.to_bf16_bits(learned.init_params(7))
    for v, t in (synth.random_triangles(65536, seed=5551), synth.noisy_icosphere(6, seed=5552)):
        plain = _sah(gpu_build(fresh_ctx, v, t))
        full = _sah(oracle.build(v, t, full_sweep=True))
        gated = _learned_build(fresh_ctx, v, t, trained, True)
        check_tree(gated["nodes"], gated["lens"], gated["perm"], synth.triangle_aabbs(v, t))
        s_g = _sah(gated)
        s_t = _sah(_learned_build(fresh_ctx, v, t, trained, False))
        s_u = _sah(_learned_build(fresh_ctx, v, t, untrained, False))
        assert s_g < plain and s_t < plain
        assert s_g <= full * 1.01
        assert (plain - s_t) > (plain - s_u)
