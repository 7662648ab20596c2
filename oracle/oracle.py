"""ctypes front end of the CPU oracle (``bvh_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: tests, ``__graft_entry__.smoke`` and the CPU
baseline leg of ``bench.py`` use it as the checker. The product path never
imports this module.

PARITY UNPINNED: the reference crate cannot be built here and ships no
golden vectors; the oracle restates ``bvh/src/lib.rs`` and is pinned by
hand-worked known-answer trees and by the reference's own invariants.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmgbvh_oracle.so")
_lock = threading.Lock()
_lib = None


class Stats(ctypes.Structure):
    """Mirror of ``mgbvh_stats`` (include/mgbvh.h)."""

    _fields_ = [
        ("construction_time", ctypes.c_double),
        ("node_count", ctypes.c_uint32),
        ("leaf_node_count", ctypes.c_uint32),
        ("min_leaf_object_count", ctypes.c_uint32),
        ("max_leaf_object_count", ctypes.c_uint32),
        ("avg_leaf_object_count", ctypes.c_double),
        ("stddev_leaf_object_count", ctypes.c_double),
        ("total_object_count", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("max_depth", ctypes.c_uint32),
        ("median_splits", ctypes.c_uint32),
        ("depth_capped_leaves", ctypes.c_uint32),
        ("feasible", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32),
        ("levels", ctypes.c_uint32),
        ("phase_seconds", ctypes.c_double * 4),
        ("graph_replay", ctypes.c_uint32),
        ("learned_splits", ctypes.c_uint32),
    ]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["phase_seconds"] = list(self.phase_seconds)
        return d


class _Knobs(ctypes.Structure):
    _fields_ = [
        ("bins", ctypes.c_uint32),
        ("adaptive_max_n", ctypes.c_uint32),
        ("adaptive_steps", ctypes.c_uint32),
        ("faithful", ctypes.c_uint32),
        ("full_sweep", ctypes.c_uint32),
        ("learn_max_n", ctypes.c_uint32),
        ("prop0", ctypes.c_uint32),
        ("prop1", ctypes.c_uint32),
    ]


def build_library(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc only; no GPU needed)."""
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
        os.path.join(_HERE, "bvh_oracle.cpp")
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH):
                build_library()
            L = ctypes.CDLL(_LIB_PATH)
            P = ctypes.c_void_p
            u32 = ctypes.c_uint32
            L.oracle_build.argtypes = [P, u32, P, P, u32, P, u32, u32, u32,
                                       ctypes.POINTER(_Knobs), P, u32, P, P,
                                       ctypes.POINTER(u32), ctypes.POINTER(Stats)]
            L.oracle_build.restype = ctypes.c_int
            L.oracle_last_tie_events.restype = u32
            L.oracle_last_order_dependent.restype = u32
            L.oracle_trace_bruteforce.argtypes = [P, u32, P, u32, P, u32, P, P]
            L.oracle_trace_bruteforce.restype = None
            L.oracle_trace_scene_bruteforce.argtypes = [P, u32, P, P, u32, P, u32, P, u32, P, P, P]
            L.oracle_trace_scene_bruteforce.restype = None
            L.oracle_sample_nodes.argtypes = [P, u32, P, u32, u32, P, u32]
            L.oracle_instance_aabbs.argtypes = [P, u32, P, P, u32, P]
            L.oracle_instance_aabbs.restype = u32
            L.oracle_sample_nodes.restype = u32
            _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build(vertices=None, triangles=None, aabbs=None, *, vertex_stride_bytes=32,
          root_bounds=None, min_leaf=1, max_leaf=1, max_depth=32, bins=0,
          adaptive_max_n=32, adaptive_steps=0, faithful=False, full_sweep=False,
          learned=None):
    """Build one BVH with the oracle.

    Either ``vertices`` (float32 [V, stride/4]) + ``triangles`` (uint32 [N, 3])
    or ``aabbs`` (float32 [N, 6]). Returns a dict with ``status``, ``nodes``
    (uint32 [count, 8], the mgbvh_node layout), ``lens``, ``perm``, ``stats``
    and ``tie_events``. ``learned`` = (max_n, proposal0, proposal1) applies the
    learned form's split rule with fixed (axis * 16 + bucket) proposals at
    every binned node of 33..max_n objects.
    """
    L = lib()
    if aabbs is not None:
        aabbs = np.ascontiguousarray(aabbs, dtype=np.float32)
        n = aabbs.shape[0]
        vp = tp = None
    else:
        vertices = np.ascontiguousarray(vertices, dtype=np.float32)
        triangles = np.ascontiguousarray(triangles, dtype=np.uint32)
        n = triangles.shape[0]
        vp, tp = vertices, triangles
    cap = max(2 * n - 1, 1)
    nodes = np.zeros((cap, 8), dtype=np.uint32)
    lens = np.zeros(cap, dtype=np.uint32)
    perm = np.zeros(max(n, 1), dtype=np.uint32)
    rb = None if root_bounds is None else np.ascontiguousarray(root_bounds, dtype=np.float32)
    count = ctypes.c_uint32(0)
    st = Stats()
    lm, p0, p1 = learned if learned is not None else (0, 0, 0)
    kn = _Knobs(bins, adaptive_max_n, adaptive_steps, 1 if faithful else 0, 1 if full_sweep else 0,
                lm, p0, p1)
    status = L.oracle_build(_ptr(vp), vertex_stride_bytes, _ptr(tp), _ptr(aabbs), n, _ptr(rb),
                            min_leaf, max_leaf, max_depth, ctypes.byref(kn), _ptr(nodes), cap,
                            _ptr(lens), _ptr(perm), ctypes.byref(count), ctypes.byref(st))
    c = count.value
    return {
        "status": status,
        "nodes": nodes[:c].copy(),
        "lens": lens[:c].copy(),
        "perm": perm[:n].copy(),
        "stats": st.as_dict(),
        "tie_events": L.oracle_last_tie_events(),
        "order_dependent": L.oracle_last_order_dependent(),
    }


def trace_bruteforce(vertices, triangles, rays):
    """Closest hit of each ray against every triangle (CPU); returns (t, prim)."""
    L = lib()
    v = np.ascontiguousarray(vertices, dtype=np.float32)
    t = np.ascontiguousarray(triangles, dtype=np.uint32)
    r = np.ascontiguousarray(rays, dtype=np.float32)
    out_t = np.zeros(r.shape[0], np.float32)
    out_p = np.zeros(r.shape[0], np.uint32)
    L.oracle_trace_bruteforce(_ptr(v), v.shape[1], _ptr(t), t.shape[0], _ptr(r), r.shape[0],
                              _ptr(out_t), _ptr(out_p))
    return out_t, out_p


def trace_scene_bruteforce(vertices, triangles, meshes, instances, rays):
    """Closest hit of each world-space ray in a two-level scene, every
    triangle of every instance tested in mesh space (CPU). vertices float32
    [V, k]; triangles uint32 [T, 3] relative to each mesh's vertex offset;
    meshes uint32 [M, 4] (BLAS root, triangle offset, count, vertex offset);
    instances [I, 20] words (inverse transform, mesh, pad). Returns (t,
    instance, triangle)."""
    L = lib()
    v = np.ascontiguousarray(vertices, dtype=np.float32)
    t = np.ascontiguousarray(triangles, dtype=np.uint32)
    m = np.ascontiguousarray(meshes).view(np.uint32)
    ins = np.ascontiguousarray(instances).view(np.uint32)
    r = np.ascontiguousarray(rays, dtype=np.float32)
    n = r.shape[0]
    out_t = np.zeros(n, np.float32)
    out_i = np.zeros(n, np.uint32)
    out_p = np.zeros(n, np.uint32)
    L.oracle_trace_scene_bruteforce(_ptr(v), v.shape[1], _ptr(t), _ptr(m), m.shape[0], _ptr(ins), ins.shape[0],
                                    _ptr(r), n, _ptr(out_t), _ptr(out_i), _ptr(out_p))
    return out_t, out_i, out_p


SAMPLE_WIDTH = 30  # 24 features, label, gain, n, plain cost, full-sweep cost, start


def sample_nodes(vertices, triangles, min_n=33):
    """Training samples of the learned split proposer from one plain build:
    float32 [K, 30] rows (features[0:24], label bits, gain, n, costs, start)."""
    L = lib()
    v = np.ascontiguousarray(vertices, dtype=np.float32)
    t = np.ascontiguousarray(triangles, dtype=np.uint32)
    cap = max(t.shape[0] // 4, 16)
    out = np.zeros((cap, SAMPLE_WIDTH), np.float32)
    k = L.oracle_sample_nodes(_ptr(v), v.shape[1] * 4, _ptr(t), t.shape[0], min_n, _ptr(out), cap)
    return out[:k].copy()


def instance_aabbs(mesh_bounds, instance_mesh, transforms):
    """World AABBs of instances (marigold/src/app/data/scene/model.rs:191-234,
    glam's Mat4 * Vec4 order): float32 [I, 6] and the count of instances whose
    mesh index is out of range."""
    L = lib()
    b = np.ascontiguousarray(mesh_bounds, dtype=np.float32)
    m = np.ascontiguousarray(instance_mesh, dtype=np.uint32)
    x = np.ascontiguousarray(transforms, dtype=np.float32)
    out = np.zeros((m.shape[0], 6), np.float32)
    bad = L.oracle_instance_aabbs(_ptr(b), b.shape[0], _ptr(m), _ptr(x), m.shape[0], _ptr(out))
    return out, bad
