"""Calls into libmgbvh.so through its C ABI for the GPU tests, with the same
argument names as the oracle's ``build`` so results compare field by field."""
from __future__ import annotations

import ctypes

import numpy as np

from marigold_b200 import _lib
from marigold_b200.bvh import NODE_DTYPE


def _vp(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def settings(root_bounds=None, min_leaf=1, max_leaf=1, max_depth=32, bins=0, adaptive_max_n=32,
             adaptive_steps=0, profiling=True):
    s = _lib.Settings()
    _lib.load().mgbvh_default_settings(ctypes.byref(s))
    s.min_leaf_objects = min_leaf
    s.max_leaf_objects = max_leaf
    s.max_depth = max_depth
    if root_bounds is not None:
        s.has_bounds = 1
        for i in range(6):
            s.bounds[i] = float(root_bounds[i])
    s.bins = bins
    s.adaptive_max_n = adaptive_max_n
    s.adaptive_steps = adaptive_steps
    s.profiling_info = 1 if profiling else 0
    return s


def gpu_build(ctx, vertices=None, triangles=None, aabbs=None, *, vertex_stride_bytes=32,
              capacity=None, **kw):
    L = ctx.L
    cs = settings(**kw)
    if aabbs is not None:
        aabbs = np.ascontiguousarray(aabbs, np.float32)
        n = aabbs.shape[0]
    else:
        vertices = np.ascontiguousarray(vertices, np.float32)
        triangles = np.ascontiguousarray(triangles, np.uint32)
        n = triangles.shape[0]
    cap = capacity if capacity is not None else max(2 * n - 1, 1)
    nodes = np.zeros(max(cap, 1), NODE_DTYPE)
    lens = np.zeros(max(cap, 1), np.uint32)
    perm = np.zeros(max(n, 1), np.uint32)
    count = ctypes.c_uint32(0)
    st = _lib.Stats()
    if aabbs is not None:
        rc = L.mgbvh_build_aabbs(ctx.ptr, _vp(aabbs), n, ctypes.byref(cs), _vp(nodes), cap,
                                 ctypes.byref(count), _vp(lens), _vp(perm), ctypes.byref(st))
    else:
        rc = L.mgbvh_build_indexed(ctx.ptr, _vp(vertices), vertex_stride_bytes,
                                   vertices.shape[0], _vp(triangles), n, ctypes.byref(cs),
                                   _vp(nodes), cap, ctypes.byref(count), _vp(lens), _vp(perm),
                                   ctypes.byref(st))
    c = count.value
    return {"status": rc, "error": ctx.last_error() if rc < 0 else "",
            "nodes": nodes[:c].view(np.uint32).reshape(-1, 8).copy(), "lens": lens[:c].copy(),
            "perm": perm[:n].copy(), "stats": st.as_dict()}
