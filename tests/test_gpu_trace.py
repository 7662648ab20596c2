"""Closest-hit traversal vs brute force (needs a B200).

The traversal of a GPU-built BVH must return, for every ray, the same hit as
testing the ray against every triangle: the same triangle index and the same
distance bit for bit (both use one triangle test; equal distances resolve to
the lowest index). The GPU brute force is itself checked against the CPU
oracle's brute force on a subset of the rays.
"""
import ctypes

import numpy as np
import pytest

from marigold_b200 import BvhSettings, _lib, build_device, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def build_and_trace(vertices, triangles, rays, brute=True, **build_kw):
    import torch
    dv = torch.from_numpy(np.ascontiguousarray(vertices)).cuda()
    dt = torch.from_numpy(np.ascontiguousarray(triangles).view(np.int32)).cuda()
    n = triangles.shape[0]
    ctx = _lib.Context(0)
    nodes = torch.zeros((2 * n - 1) * 8, dtype=torch.int32, device="cuda")
    lens = torch.zeros(2 * n - 1, dtype=torch.int32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    count, rc, _ = build_device(ctx, BvhSettings(), nodes, perm, vertices=dv, triangles=dt,
                                out_lens=lens, **build_kw)
    assert rc >= 0
    torch.cuda.synchronize()
    tr = _lib.Tracer(0)
    L = tr.L
    stream = torch.cuda.current_stream().cuda_stream
    use_lens = build_kw.get("max_leaf_objects", 1) > 1
    tr.check(L.mgbvh_tracer_set_blas_dev(tr.ptr, _vp(nodes), count, _vp(lens) if use_lens else None,
                                         _vp(dv), vertices.shape[1] * 4, vertices.shape[0], _vp(dt),
                                         _vp(perm), n, ctypes.c_void_p(stream)))
    dr = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    m = rays.shape[0]
    ht = torch.zeros(m, dtype=torch.float32, device="cuda")
    hp = torch.zeros(m, dtype=torch.int32, device="cuda")
    counts = (ctypes.c_uint64 * 3)()
    secs = ctypes.c_double(0)
    tr.check(L.mgbvh_trace_closest_dev(tr.ptr, _vp(dr), m, _vp(ht), _vp(hp), counts,
                                       ctypes.byref(secs), ctypes.c_void_p(stream)))
    out = {"t": ht.cpu().numpy(), "prim": hp.cpu().numpy().view(np.uint32),
           "counts": list(counts), "seconds": secs.value}
    if brute:
        bt = torch.zeros(m, dtype=torch.float32, device="cuda")
        bp = torch.zeros(m, dtype=torch.int32, device="cuda")
        tr.check(L.mgbvh_trace_bruteforce_dev(tr.ptr, _vp(dr), m, _vp(bt), _vp(bp),
                                              ctypes.c_void_p(stream)))
        out["bt"] = bt.cpu().numpy()
        out["bp"] = bp.cpu().numpy().view(np.uint32)
    tr.close()
    ctx.close()
    return out


def assert_same_hits(t1, p1, t2, p2):
    bad = np.nonzero((p1 != p2) | (t1.view(np.uint32) != t2.view(np.uint32)))[0]
    assert bad.size == 0, (f"{bad.size} rays differ, first {bad[0]}: "
                           f"({t1[bad[0]]}, {p1[bad[0]]}) vs ({t2[bad[0]]}, {p2[bad[0]]})")


@pytest.mark.parametrize("max_leaf", [1, 4])
def test_traversal_equals_bruteforce_mixed_scene(max_leaf):
    v, t = synth.mixed_scene(seed=11, n_blob=40000, grid=(128, 64), n_thin=20000)
    rays = synth.rays_in_box(8192, v.min(0), v.max(0), seed=12)
    kw = {} if max_leaf == 1 else dict(min_leaf_objects=1, max_leaf_objects=max_leaf)
    r = build_and_trace(v, t, rays, **kw)
    assert (r["bp"] != 0xFFFFFFFF).sum() > 1000  # the rays do hit things
    assert_same_hits(r["t"], r["prim"], r["bt"], r["bp"])


def test_gpu_bruteforce_equals_cpu_bruteforce():
    v, t = synth.mixed_scene(seed=13, n_blob=20000, grid=(64, 32), n_thin=8000)
    rays = synth.rays_in_box(256, v.min(0), v.max(0), seed=14)
    r = build_and_trace(v, t, rays)
    ct, cp = orc.trace_bruteforce(v, t, rays)
    assert_same_hits(r["bt"], r["bp"], ct, cp)
    assert_same_hits(r["t"], r["prim"], ct, cp)


def test_traversal_icosphere_rays_from_inside():
    v, t = synth.noisy_icosphere(5, seed=3)
    pos = v[:, 0:3].copy()
    rays = synth.rays_in_box(4096, [-0.5] * 3, [0.5] * 3, seed=15, expand=0.0)
    r = build_and_trace(pos, t, rays)
    # rays from inside a closed sphere hit it (a ray through an edge may slip
    # between the two triangles' rounded tests)
    assert (r["prim"] != 0xFFFFFFFF).mean() > 0.999
    assert_same_hits(r["t"], r["prim"], r["bt"], r["bp"])
    nodes, boxes, tris = r["counts"]
    assert nodes > 0 and boxes > 0 and tris > 0
