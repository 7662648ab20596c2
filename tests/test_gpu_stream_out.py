"""Host-pointer builds into page-locked output arrays (needs a B200).

When the caller's node (and lens) arrays are page-locked and hold every
slot, a build with one object per leaf sends the nodes to the host in slot
chunks while its subtree kernels still run. These tests check that such a
build returns the same bytes as the same build into pageable arrays (which
copies after the build) and as the oracle, including the cases that fall
back to copying after the build: leaves of several objects, depth-capped
leaves (compacted slots), no lens array.
"""
import ctypes

import numpy as np
import pytest

from marigold_b200 import _lib, synth
from tests.gpuhelp import settings
from tests.treecheck import compare_exact

pytestmark = pytest.mark.gpu


def _host_arrays(n, pinned, with_lens):
    cap = 2 * n - 1
    if pinned:
        import torch
        nodes_t = torch.zeros(cap * 8, dtype=torch.int32).pin_memory()
        perm_t = torch.zeros(n, dtype=torch.int32).pin_memory()
        lens_t = torch.zeros(cap, dtype=torch.int32).pin_memory() if with_lens else None
        keep = (nodes_t, perm_t, lens_t)
        nodes = nodes_t.numpy().view(np.uint32).reshape(cap, 8)
        perm = perm_t.numpy().view(np.uint32)
        lens = lens_t.numpy().view(np.uint32) if with_lens else None
    else:
        keep = ()
        nodes = np.zeros((cap, 8), np.uint32)
        perm = np.zeros(n, np.uint32)
        lens = np.zeros(cap, np.uint32) if with_lens else None
    return keep, nodes, lens, perm


def _vp(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def host_build(ctx, v=None, t=None, aabbs=None, *, pinned, with_lens=True, **kw):
    n = aabbs.shape[0] if aabbs is not None else t.shape[0]
    keep, nodes, lens, perm = _host_arrays(n, pinned, with_lens)
    cs = settings(profiling=False, **kw)
    count = ctypes.c_uint32(0)
    st = _lib.Stats()
    if aabbs is not None:
        a = np.ascontiguousarray(aabbs, np.float32)
        rc = ctx.L.mgbvh_build_aabbs(ctx.ptr, _vp(a), n, ctypes.byref(cs), _vp(nodes), 2 * n - 1,
                                     ctypes.byref(count), _vp(lens), _vp(perm), ctypes.byref(st))
    else:
        rc = ctx.L.mgbvh_build_indexed(ctx.ptr, _vp(v), 4 * v.shape[1], v.shape[0], _vp(t), n,
                                       ctypes.byref(cs), _vp(nodes), 2 * n - 1, ctypes.byref(count),
                                       _vp(lens), _vp(perm), ctypes.byref(st))
    assert rc == 0, ctx.last_error()
    c = count.value
    out = {"nodes": nodes[:c].copy(), "lens": None if lens is None else lens[:c].copy(),
           "perm": perm.copy(), "count": c, "launches": st.as_dict()["kernel_launches"]}
    del keep
    return out


def _same(a, b):
    assert a["count"] == b["count"]
    assert np.array_equal(a["nodes"], b["nodes"])
    assert np.array_equal(a["perm"], b["perm"])
    if a["lens"] is not None and b["lens"] is not None:
        assert np.array_equal(a["lens"], b["lens"])


@pytest.mark.parametrize("n", [3000, 200000])
def test_streamed_equals_pageable_and_oracle(oracle, gpu_ctx, n):
    """n = 3000: the root is one subtree CTA; n = 200000: level passes first.
    The streamed build runs a count and a sort of the subtree CTA tasks, then
    per slot chunk a subtree CTA launch, a selection and a small-kernel launch:
    26 launches in place of 2 (kernel_launches shows the streamed path ran)."""
    v, t = synth.random_triangles(n, seed=300 + n)
    host_build(gpu_ctx, v, t, pinned=False)  # the context's level-count hint now fits this mesh
    p = host_build(gpu_ctx, v, t, pinned=True)
    q = host_build(gpu_ctx, v, t, pinned=False)
    _same(p, q)
    assert p["launches"] == q["launches"] + 24
    o = oracle.build(v, t)
    assert compare_exact(p["nodes"], p["lens"], p["perm"], o["nodes"], o["lens"], o["perm"]) is None


def test_streamed_without_lens(gpu_ctx):
    v, t = synth.random_triangles(120000, seed=41)
    host_build(gpu_ctx, v, t, pinned=False)
    p = host_build(gpu_ctx, v, t, pinned=True, with_lens=False)
    q = host_build(gpu_ctx, v, t, pinned=False)
    _same(p, q)
    assert p["launches"] == q["launches"] + 24


@pytest.mark.parametrize("kw", [dict(max_depth=9), dict(min_leaf=1, max_leaf=4)])
def test_fallbacks_equal_oracle(oracle, gpu_ctx, kw):
    """Depth-capped leaves hold several objects, so slots are compacted after
    the build and the streamed chunks are replaced; leaves of up to four
    objects do not stream at all."""
    v, t = synth.random_triangles(60000, seed=43)
    p = host_build(gpu_ctx, v, t, pinned=True, **kw)
    q = host_build(gpu_ctx, v, t, pinned=False, **kw)
    _same(p, q)
    o = oracle.build(v, t, **kw)
    assert compare_exact(p["nodes"], p["lens"], p["perm"], o["nodes"], o["lens"], o["perm"]) is None


def test_streamed_aabbs_and_repeated_calls(gpu_ctx):
    """The bounding-volume entry point, and calls in a row on one context
    whose trees differ in size (a chunk of an earlier tree must not survive)."""
    v1, t1 = synth.random_triangles(90000, seed=51)
    v2, t2 = synth.random_triangles(150000, seed=52)
    a1 = synth.triangle_aabbs(v1, t1)
    for kind in range(2):
        for v, t in ((v1, t1), (v2, t2), (v1, t1)):
            if kind == 0:
                p = host_build(gpu_ctx, v, t, pinned=True)
                q = host_build(gpu_ctx, v, t, pinned=False)
            else:
                a = a1 if v is v1 else synth.triangle_aabbs(v, t)
                p = host_build(gpu_ctx, aabbs=a, pinned=True)
                q = host_build(gpu_ctx, aabbs=a, pinned=False)
            _same(p, q)
