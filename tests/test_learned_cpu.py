"""CPU checks of the learned split proposer's checkers and host code: the
oracle's node samples (features, full-sweep labels), the float64 MLP
reference's gradient against finite differences, and the BF16 packing the
training loop uses."""
from __future__ import annotations

import numpy as np
import pytest

from marigold_b200 import learned, synth


@pytest.fixture(scope="module")
def mlp_ref():
    from oracle import mlp_ref as m
    return m


def test_sample_nodes_invariants(oracle):
    v, t = synth.random_triangles(3000, seed=31)
    s = oracle.sample_nodes(v, t, min_n=33)
    assert s.shape[1] == oracle.SAMPLE_WIDTH == learned.SAMPLE_WIDTH == 30
    assert s.shape[0] > 50
    f = s[:, :24]
    assert np.all(np.isfinite(f))
    assert np.all((f[:, 0:6] >= 0) & (f[:, 0:6] <= 1))
    # 4-bucket histograms sum to 1 on every axis with a centroid extent
    for a in range(3):
        h = f[:, 7 + 4 * a:11 + 4 * a].sum(axis=1)
        has = f[:, 3 + a] > 0
        assert np.allclose(h[has], 1.0, atol=1e-5)
    lab = s[:, 24].view(np.uint32)
    n = s[:, 26]
    plain, full = s[:, 27], s[:, 28]
    ok = lab != 0xFFFFFFFF
    assert np.all(lab[ok] < 48)
    assert np.all(n >= 33)
    # a binned split is a threshold split on centroids: the exact sweep over
    # every centroid can only be as good or better
    fin = np.isfinite(plain)
    assert np.all(full[fin] <= plain[fin])
    assert np.array_equal(s[ok & fin, 25] == 1.0, full[ok & fin] < plain[ok & fin])
    start = s[:, 29].astype(np.int64)
    assert np.all(start + n.astype(np.int64) <= t.shape[0])
    assert start[0] == 0 and n[0] == t.shape[0]  # the root comes first


def test_sample_known_split(oracle):
    """Two clusters on x, 40 and 24 triangles far apart: the exact optimum is
    the gap between them on axis 0, at position bucket floor(16 * c / ext)."""
    tris = []
    rng = np.random.default_rng(5)
    for cx, k in ((0.0, 40), (10.0, 24)):
        for _ in range(k):
            p = np.array([cx, 0.0, 0.0]) + rng.uniform(0, 0.5, 3)
            tris.append([p, p + [0.01, 0, 0], p + [0, 0.01, 0.01]])
    pos = np.array(tris, np.float64).reshape(-1, 3)
    v = synth.pack_vertices(pos)
    t = np.arange(pos.shape[0], dtype=np.uint32).reshape(-1, 3)
    s = oracle.sample_nodes(v, t, min_n=64)
    assert s.shape[0] == 1
    lab = int(s[0, 24].view(np.uint32))
    assert lab // 16 == 0
    # the split threshold is the smallest centroid of the far cluster: the
    # last bucket of the centroid extent
    assert lab % 16 == 15
    assert s[0, 26] == 64


def test_mlp_ref_gradient_matches_finite_differences(mlp_ref):
    rng = np.random.default_rng(0)
    p = learned.init_params(1).astype(np.float64)
    B = 6
    x = rng.normal(size=(B, 24))
    label = rng.integers(0, 48, B).astype(np.uint32)
    label[2] = mlp_ref.NO_LABEL
    gain = (rng.random(B) < 0.5).astype(np.float64)
    _, g = mlp_ref.loss_and_grad(p, x, label, gain)
    idx = np.concatenate([rng.choice(np.arange(s, e), 6, replace=False) for s, e in (
        (0, 1536), (1536, 1600), (1600, 5696), (5696, 5760), (5760, 8896), (8896, 8945))])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        num = (mlp_ref.loss_and_grad(pp, x, label, gain)[0] -
               mlp_ref.loss_and_grad(pm, x, label, gain)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, num, g[i])


def test_bf16_packing(mlp_ref):
    rng = np.random.default_rng(2)
    p = np.concatenate([rng.normal(size=1000).astype(np.float32),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, -3.5e-3], np.float32)])
    bits = learned.to_bf16_bits(p)
    back = (bits.astype(np.uint32) << 16).view(np.float32)
    assert np.array_equal(back, mlp_ref.bf16_round(p))
    # ties to even: 1 + 2^-8 rounds down to 1, 1 + 3 * 2^-8 rounds up
    assert back[1003] == 1.0 and back[1004] == np.float32(1.015625)


def test_init_params_layout():
    p = learned.init_params(3)
    assert p.shape == (learned.NPARAM,) and p.dtype == np.float32
    assert np.all(np.abs(p[0:1536]) <= 1 / np.sqrt(24) + 1e-7)
    assert np.all(np.abs(p[5760:8896]) <= 1 / 8 + 1e-7)
    assert np.count_nonzero(p) == learned.NPARAM


def test_oracle_learned_form_valid(oracle):
    """The oracle's restatement of the learned split rule (fixed proposals)
    builds valid trees and replaces some binned splits."""
    from tests.treecheck import check_tree
    v, t = synth.random_triangles(20000, seed=91)
    r = oracle.build(v, t, learned=(1024, 7, 23))
    assert r["status"] == 0 and r["stats"]["learned_splits"] > 0
    check_tree(r["nodes"], r["lens"], r["perm"], synth.triangle_aabbs(v, t))
    # proposals at the far ends of the extent never beat the binned split
    r2 = oracle.build(v, t, learned=(1024, 15, 31))
    assert r2["stats"]["learned_splits"] == 0
    plain = oracle.build(v, t)
    assert np.array_equal(r2["nodes"], plain["nodes"])
