"""The allocation-free build entry point (mgbvh_build_aabbs_noalloc).

Some callers may not allocate while they build: a render loop that rebuilds
its TLAS every frame cannot call cudaMalloc/cudaFree there (they can
synchronize the whole device), and an engine that owns all device memory
through its own pool may not allocate behind its back. This entry point
takes device buffers from the caller and keeps its scratch in a fixed array
inside the library, so it allocates nothing.

Checked here through the C ABI: two calls in a row, each bit-exact against
the allocating entry point (mgbvh_build_aabbs) on the same input. The file
is named so pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from marigold_b200 import _lib
from marigold_b200.bvh import NODE_DTYPE
from tests.gpuhelp import gpu_build, settings
from tests.treecheck import compare_exact

pytestmark = pytest.mark.gpu


def boxes(n, seed):
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-100, 100, size=(n, 3)).astype(np.float32)
    ext = rng.uniform(0.5, 20, size=(n, 3)).astype(np.float32)
    return np.concatenate([lo, lo + ext], axis=1)


def noalloc_build(aabbs, **kw):
    import torch
    L = _lib.load()
    n = aabbs.shape[0]
    cap = max(2 * n - 1, 1)
    d_aabbs = torch.from_numpy(aabbs).cuda()
    d_nodes = torch.zeros(cap * 8, dtype=torch.int32, device="cuda")
    d_lens = torch.zeros(cap, dtype=torch.int32, device="cuda")
    d_perm = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    cs = settings(**kw)
    count = ctypes.c_uint32(0)
    torch.cuda.synchronize()
    rc = L.mgbvh_build_aabbs_noalloc(
        ctypes.c_void_p(d_aabbs.data_ptr()), n, ctypes.byref(cs),
        ctypes.c_void_p(d_nodes.data_ptr()), cap, ctypes.byref(count),
        ctypes.c_void_p(d_lens.data_ptr()), ctypes.c_void_p(d_perm.data_ptr()), None)
    c = count.value
    return {"status": rc,
            "nodes": d_nodes.cpu().numpy().view(np.uint32).reshape(-1, 8)[:c],
            "lens": d_lens.cpu().numpy().view(np.uint32)[:c],
            "perm": d_perm.cpu().numpy().view(np.uint32)[:n]}


def test_two_calls_in_a_row_match_the_allocating_build():
    ctx = _lib.Context(0)
    cases = [(boxes(1000, 1), {}), (boxes(300, 2), dict(min_leaf=2, max_leaf=4))]
    for aabbs, kw in cases:
        got = noalloc_build(aabbs, **kw)
        want = gpu_build(ctx, aabbs=aabbs, **kw)
        assert got["status"] == want["status"] >= 0, (got["status"], want["status"], want["error"])
        msg = compare_exact(got["nodes"], got["lens"], got["perm"], want["nodes"], want["lens"],
                            want["perm"])
        assert msg is None, msg
    ctx.close()


def test_rejects_more_than_the_limit():
    got = noalloc_build(boxes(_lib.NOALLOC_MAX_OBJECTS + 1, 3))
    assert got["status"] == _lib.ERR_TOO_LARGE


@pytest.mark.parametrize("n", [1, 2, 32, 33, 1024])
def test_sizes_against_the_oracle(oracle, n):
    """n = 1: the root is a leaf; 2 and 32: one warp subtree; 33: the
    smallest subtree-CTA build; 1024: the limit. Each equals the oracle and
    the allocating build, in both leaf-size profiles."""
    ctx = _lib.Context(0)
    for kw in ({}, dict(min_leaf=2, max_leaf=4)):
        aabbs = boxes(n, 40 + n)
        got = noalloc_build(aabbs, **kw)
        want = oracle.build(aabbs=aabbs, **kw)
        assert got["status"] == want["status"] >= 0, (n, kw, got["status"], want["status"])
        msg = compare_exact(got["nodes"], got["lens"], got["perm"], want["nodes"], want["lens"], want["perm"])
        assert msg is None, (n, kw, msg)
        alloc = gpu_build(ctx, aabbs=aabbs, **kw)
        msg = compare_exact(got["nodes"], got["lens"], got["perm"], alloc["nodes"], alloc["lens"], alloc["perm"])
        assert msg is None, (n, kw, msg)
    ctx.close()


def test_capacity_too_small():
    import torch
    L = _lib.load()
    aabbs = boxes(500, 7)
    n = aabbs.shape[0]
    cap = 2 * n - 2  # one node short of the tree
    d_aabbs = torch.from_numpy(aabbs).cuda()
    d_nodes = torch.zeros(cap * 8, dtype=torch.int32, device="cuda")
    d_perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    count = ctypes.c_uint32(12345)
    torch.cuda.synchronize()
    rc = L.mgbvh_build_aabbs_noalloc(ctypes.c_void_p(d_aabbs.data_ptr()), n, ctypes.byref(settings()),
                                     ctypes.c_void_p(d_nodes.data_ptr()), cap, ctypes.byref(count), None,
                                     ctypes.c_void_p(d_perm.data_ptr()), None)
    assert rc == _lib.ERR_CAPACITY and count.value == 0
    # the next call on the shared scratch is unaffected
    got = noalloc_build(aabbs)
    assert got["status"] == 0 and got["nodes"].shape[0] == 2 * n - 1
