"""The 8-wide BVH with quantized child boxes, collapsed on the GPU from the
builder's binary tree: closest hits through it equal the binary traversal's
and brute force's bit for bit; every triangle sits in exactly one leaf child;
every dequantized box on a triangle's path contains the triangle's box."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from marigold_b200 import _lib, synth

from tests.gpuhelp import gpu_build

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

WNODE = np.dtype([("p", "<f4", 3), ("e", "u1", 3), ("n", "u1"), ("qlo", "u1", (3, 8)),
                  ("qhi", "u1", (3, 8)), ("ref", "<u4", 8), ("cnt", "u1", 8), ("pad", "<u4", 2)])
assert WNODE.itemsize == 112


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _setup(ctx, v, t, **kw):
    r = gpu_build(ctx, v, t, **kw)
    assert r["status"] >= 0, r["error"]
    tr = _lib.Tracer(0)
    L = tr.L
    dn = torch.from_numpy(r["nodes"].view(np.int32).reshape(-1)).cuda()
    dl = torch.from_numpy(r["lens"].view(np.int32)).cuda()
    dv = torch.from_numpy(v).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    dp = torch.from_numpy(r["perm"].view(np.int32)).cuda()
    s = torch.cuda.current_stream().cuda_stream
    multi = int(r["lens"][r["nodes"][:, 7] == 0].max()) > 1
    tr.check(L.mgbvh_tracer_set_blas_dev(tr.ptr, _vp(dn), r["nodes"].shape[0], _vp(dl) if multi else None,
                                         _vp(dv), v.shape[1] * 4, v.shape[0], _vp(dt), _vp(dp), t.shape[0],
                                         ctypes.c_void_p(s)))
    cnt = ctypes.c_uint32(0)
    tr.check(L.mgbvh_tracer_build_wide(tr.ptr, ctypes.c_void_p(s), ctypes.byref(cnt)))
    return tr, r, (dn, dl, dv, dt, dp), cnt.value


def _trace(tr, fn, dr, m):
    L = tr.L
    ht = torch.empty(m, dtype=torch.float32, device="cuda")
    hp = torch.empty(m, dtype=torch.int32, device="cuda")
    counts = (ctypes.c_uint64 * 3)()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if fn == "brute":
        tr.check(L.mgbvh_trace_bruteforce_dev(tr.ptr, _vp(dr), m, _vp(ht), _vp(hp), s))
    else:
        f = L.mgbvh_trace_closest_wide_dev if fn == "wide" else L.mgbvh_trace_closest_dev
        tr.check(f(tr.ptr, _vp(dr), m, _vp(ht), _vp(hp), counts, None, s))
    torch.cuda.synchronize()
    return ht.cpu().numpy(), hp.cpu().numpy().view(np.uint32), list(counts)


CASES = {
    "random50k": lambda: (synth.random_triangles(50000, seed=61), {}),
    "icosphere6": lambda: (synth.noisy_icosphere(6, seed=62), {}),
    "leaves_of_4": lambda: (synth.random_triangles(30000, seed=63), {"min_leaf": 1, "max_leaf": 4}),
    "depth_capped": lambda: (synth.random_triangles(20000, seed=64), {"max_depth": 9}),
    "one_triangle": lambda: (synth.random_triangles(1, seed=65), {}),
}


@pytest.mark.parametrize("case", list(CASES))
def test_wide_hits_equal_binary_and_bruteforce(gpu_ctx, case):
    (v, t), kw = CASES[case]()
    tr, r, keep, wcount = _setup(gpu_ctx, v, t, **kw)
    assert 1 <= wcount <= r["nodes"].shape[0]
    rays = synth.rays_in_box(4096, v[:, :3].min(0), v[:, :3].max(0), seed=66)
    dr = torch.from_numpy(rays).cuda()
    wt, wp, wc = _trace(tr, "wide", dr, 4096)
    bt, bp, bc = _trace(tr, "binary", dr, 4096)
    xt, xp, _ = _trace(tr, "brute", dr, 4096)
    assert np.array_equal(wp, xp) and np.array_equal(wt.view(np.uint32), xt.view(np.uint32))
    assert np.array_equal(bp, xp) and np.array_equal(bt.view(np.uint32), xt.view(np.uint32))
    assert (xp != 0xFFFFFFFF).any()
    if t.shape[0] > 1000:
        assert wc[0] < bc[0]  # fewer nodes visited than the binary tree
    tr.close()


@pytest.mark.parametrize("case", ["random50k", "leaves_of_4", "depth_capped"])
def test_wide_structure(gpu_ctx, case):
    (v, t), kw = CASES[case]()
    tr, r, keep, wcount = _setup(gpu_ctx, v, t, **kw)
    ptr = ctypes.c_void_p()
    cnt = ctypes.c_uint32(0)
    tr.check(tr.L.mgbvh_tracer_wide_nodes(tr.ptr, ctypes.byref(ptr), ctypes.byref(cnt)))
    assert cnt.value == wcount
    from cuda.bindings import runtime as rt
    host = np.zeros(wcount * 112, np.uint8)
    torch.cuda.synchronize()
    err, = rt.cudaMemcpy(host.ctypes.data, ptr.value, wcount * 112, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    wn = host.view(WNODE)
    aabbs = synth.triangle_aabbs(v, t)[r["perm"]]  # triangles in leaf order
    seen = np.zeros(t.shape[0], np.int64)
    stack = [(0, np.array([-np.inf] * 3, np.float32), np.array([np.inf] * 3, np.float32))]
    while stack:
        ni, plo, phi = stack.pop()
        nd = wn[ni]
        step = (nd["e"].astype(np.uint32) << 23).view(np.float32)
        for j in range(nd["n"]):
            lo = (nd["p"] + nd["qlo"][:, j].astype(np.float32) * step).astype(np.float32)
            hi = (nd["p"] + nd["qhi"][:, j].astype(np.float32) * step).astype(np.float32)
            lo, hi = np.maximum(lo, plo), np.minimum(hi, phi)  # the path's intersection
            ref = int(nd["ref"][j])
            if ref & 0x80000000:
                s0, c = ref & 0x7FFFFFFF, int(nd["cnt"][j])
                seen[s0:s0 + c] += 1
                box = aabbs[s0:s0 + c]
                assert np.all(box[:, :3] >= lo) and np.all(box[:, 3:] <= hi), (ni, j)
            else:
                assert 0 < ref < wcount
                stack.append((ref, lo, hi))
    assert np.all(seen == 1)
    tr.close()
