"""Host-side mirror of marigold's `bvh` crate interface over the CUDA builder.

Same names and meaning as bvh/src/lib.rs:
  BoundingVolume            bvh/src/lib.rs:41-111
  BvhSettings               bvh/src/lib.rs:668-674 (plus split knobs whose
                            defaults are the reference's hard-wired values)
  BoundingVolumeHierarchy   bvh/src/lib.rs:691-887; ``new`` permutes the
                            object list in place and returns the hierarchy,
                            ``nodes()`` / ``into_nodes()`` give the node array
  BvhProfilingInfo          bvh/src/lib.rs:676-689, written as JSON the way
                            :851-867 writes it

Error behaviour follows the reference: an empty list gives an empty
hierarchy with a warning (:703-708), infeasible leaf bounds log a warning
(:716-726), and conditions the reference asserts on raise ``MgbvhError``.
Every build runs on the GPU through libmgbvh.so; nothing here computes a tree.
"""
from __future__ import annotations

import ctypes
import json
import logging
import os
import random
import threading
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import Context, MgbvhError

log = logging.getLogger("marigold_b200.bvh")

NODE_DTYPE = np.dtype([("min", "<f4", (3,)), ("start_index", "<u4"), ("max", "<f4", (3,)),
                       ("child_node", "<u4")])
assert NODE_DTYPE.itemsize == 32

DEPTH_COST = 1.0   # bvh/src/lib.rs:217
OBJECT_COST = 8.0  # bvh/src/lib.rs:218


@dataclass
class BoundingVolume:
    min: np.ndarray
    max: np.ndarray

    def as_array(self) -> np.ndarray:
        return np.concatenate([np.asarray(self.min, np.float32).reshape(3),
                               np.asarray(self.max, np.float32).reshape(3)])


@dataclass
class BvhSettings:
    name: str = "bvh"
    bounds: Optional[object] = None  # BoundingVolume or 6 floats (min xyz, max xyz)
    max_depth: int = 32
    profiling_info: bool = False
    profiling_info_directory: Optional[str] = None
    # split knobs; the defaults are the reference's fixed behaviour
    bins: int = 0
    adaptive_max_n: int = 32
    adaptive_steps: int = 0

    def to_c(self, min_leaf: int, max_leaf: int) -> _lib.Settings:
        s = _lib.Settings()
        _lib.load().mgbvh_default_settings(ctypes.byref(s))
        s.min_leaf_objects = min_leaf
        s.max_leaf_objects = max_leaf
        s.max_depth = self.max_depth
        if self.bounds is not None:
            b = self.bounds.as_array() if isinstance(self.bounds, BoundingVolume) else \
                np.asarray(self.bounds, np.float32).reshape(6)
            s.has_bounds = 1
            for i in range(6):
                s.bounds[i] = float(b[i])
        s.bins = self.bins
        s.adaptive_max_n = self.adaptive_max_n
        s.adaptive_steps = self.adaptive_steps
        s.profiling_info = 1 if self.profiling_info else 0
        return s


_tls = threading.local()


def default_context(device: int = 0) -> Context:
    """One context per thread and device (a context is not thread-safe)."""
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


def _vp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class BoundingVolumeHierarchy:
    """Result of a build: the node array (and per-node object counts)."""

    def __init__(self, nodes: np.ndarray, lens: np.ndarray, min_leaf_objects: int = 1,
                 max_leaf_objects: int = 1, stats: Optional[dict] = None,
                 status: int = _lib.OK):
        self._nodes = nodes
        self.lens = lens
        self.min_leaf_objects = min_leaf_objects
        self.max_leaf_objects = max_leaf_objects
        self.stats = stats or {}
        self.status = status

    @classmethod
    def new(cls, list, source, settings: BvhSettings, *, min_leaf_objects: int = 1,
            max_leaf_objects: int = 1, context: Optional[Context] = None):
        """BoundingVolumeHierarchy::<MIN, MAX>::new(list, source, settings).

        ``list`` is permuted in place, as the crate does. Two object kinds:
          * triangles: ``list`` uint32 [N, 3] (MeshTriangle) with ``source``
            float32 [V, k >= 3] vertex records (MeshVertex is k = 8);
          * bounding volumes: ``list`` float32 [N, 6] (min xyz, max xyz) and
            ``source`` None or empty — the AsBoundingVolume path (TLAS).
        """
        ctx = context or default_context()
        L = ctx.L
        arr = list
        n = int(arr.shape[0])
        cs = settings.to_c(min_leaf_objects, max_leaf_objects)
        cap = max(2 * n - 1, 1)
        nodes = np.zeros(cap, dtype=NODE_DTYPE)
        lens = np.zeros(cap, dtype=np.uint32)
        perm = np.zeros(max(n, 1), dtype=np.uint32)
        count = ctypes.c_uint32(0)
        st = _lib.Stats()
        triangles = source is not None and len(source) > 0
        if triangles:
            verts = np.ascontiguousarray(source, dtype=np.float32)
            tris = np.ascontiguousarray(arr, dtype=np.uint32)
            if tris.ndim != 2 or tris.shape[1] != 3:
                raise ValueError("triangle list must be uint32 [N, 3]")
            rc = L.mgbvh_build_indexed(ctx.ptr, _vp(verts), verts.shape[1] * 4, verts.shape[0],
                                       _vp(tris), n, ctypes.byref(cs), _vp(nodes), cap,
                                       ctypes.byref(count), _vp(lens), _vp(perm), ctypes.byref(st))
        else:
            boxes = np.ascontiguousarray(arr, dtype=np.float32)
            if boxes.ndim != 2 or boxes.shape[1] != 6:
                raise ValueError("bounding-volume list must be float32 [N, 6]")
            rc = L.mgbvh_build_aabbs(ctx.ptr, _vp(boxes), n, ctypes.byref(cs), _vp(nodes), cap,
                                     ctypes.byref(count), _vp(lens), _vp(perm), ctypes.byref(st))
        ctx.check(rc)
        if rc == _lib.WARN_EMPTY:
            log.warning("tried constructing a BVH with an empty object list, returning an empty BVH")
        elif rc == _lib.WARN_INFEASIBLE:
            log.warning(
                "BVH may be impossible to construct with the given constraints; min leaf objects %d "
                "and max leaf objects %d is likely impossible with total objects %d.",
                min_leaf_objects, max_leaf_objects, n)
        c = count.value
        if n > 0:
            arr[...] = arr[perm[:n]]  # the crate's in-place permutation of `list`
        stats = st.as_dict()
        bvh = cls(nodes[:c].copy(), lens[:c].copy(), min_leaf_objects, max_leaf_objects, stats, rc)
        bvh.perm = perm[:n].copy()
        if n > 0:
            if settings.profiling_info:
                log.info("BVH %s: %d objects, %d nodes, height %d, %.6f s", settings.name, n, c,
                         stats["height"], stats["construction_time"])
                if settings.profiling_info_directory:
                    write_profiling_info(settings, stats)
            else:
                log.info("BVH for %s took %s seconds to build", settings.name,
                         stats["construction_time"])
        return bvh

    def nodes(self) -> np.ndarray:
        return self._nodes

    def into_nodes(self) -> np.ndarray:
        return self._nodes

    def gpu_bytes(self) -> np.ndarray:
        """AsGpuBytes of every node (bvh/src/lib.rs:157-212): uint32 [count, 8]."""
        return encode_gpu_bytes(self._nodes, self.lens, self.max_leaf_objects)

    def sah_cost(self) -> float:
        return sah_cost(self._nodes, self.lens)


def write_profiling_info(settings: BvhSettings, stats: dict) -> str:
    """BvhProfilingInfo as JSON, one file per build (bvh/src/lib.rs:836-867)."""
    os.makedirs(settings.profiling_info_directory, exist_ok=True)
    build_id = random.randint(100000000, 999999999)
    path = os.path.join(settings.profiling_info_directory, f"bvh_{settings.name}_{build_id}.json")
    info = {
        "name": settings.name,
        "construction_time": stats["construction_time"],
        "node_count": stats["node_count"],
        "leaf_node_count": stats["leaf_node_count"],
        "min_leaf_object_count": stats["min_leaf_object_count"],
        "max_leaf_object_count": stats["max_leaf_object_count"],
        "avg_leaf_object_count": stats["avg_leaf_object_count"],
        "stddev_leaf_object_count": stats["stddev_leaf_object_count"],
        "total_object_count": stats["total_object_count"],
        "height": stats["height"],
        "max_depth": stats["max_depth"],
    }
    if not os.path.exists(path):
        with open(path, "w") as f:
            f.write(json.dumps(info) + "\n")
    return path


def encode_gpu_bytes(nodes: np.ndarray, lens: np.ndarray, max_leaf_objects: int) -> np.ndarray:
    nodes = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    out = np.zeros((nodes.shape[0], 8), dtype=np.uint32)
    rc = _lib.load().mgbvh_encode_gpu_bytes(_vp(nodes), _vp(lens), nodes.shape[0],
                                            max_leaf_objects, _vp(out))
    if rc < 0:
        raise MgbvhError(rc, "AsGpuBytes: leaf length does not fit the packed bits")
    return out


def sah_cost(nodes: np.ndarray, lens: np.ndarray) -> float:
    nodes = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
    lens = np.ascontiguousarray(lens, dtype=np.uint32)
    return float(_lib.load().mgbvh_sah_cost(_vp(nodes), _vp(lens), nodes.shape[0]))


def build_device(ctx: Context, settings: BvhSettings, out_nodes, out_perm, *, vertices=None,
                 triangles=None, aabbs=None, out_lens=None, min_leaf_objects: int = 1,
                 max_leaf_objects: int = 1, stream=None):
    """Build from device-resident torch tensors into device-resident outputs.

    vertices float32 [V, k] + triangles int32/uint32 [N, 3], or aabbs float32
    [N, 6]; out_nodes uint8/int32 tensor of >= 32*(2N-1) bytes, out_perm
    int32 [N], out_lens int32 [2N-1] or None. Runs on ``stream`` (a
    torch.cuda.Stream) or torch's current stream. Returns (count, status, stats).
    """
    import torch

    L = ctx.L
    s = stream if stream is not None else torch.cuda.current_stream()
    ctx.set_stream(s.cuda_stream)
    cs = settings.to_c(min_leaf_objects, max_leaf_objects)
    count = ctypes.c_uint32(0)
    st = _lib.Stats()
    cap = out_nodes.numel() * out_nodes.element_size() // 32
    lens_p = ctypes.c_void_p(out_lens.data_ptr()) if out_lens is not None else None
    if aabbs is None:
        n = triangles.shape[0]
        rc = L.mgbvh_build_indexed_dev(
            ctx.ptr, ctypes.c_void_p(vertices.data_ptr()), vertices.shape[1] * 4, vertices.shape[0],
            ctypes.c_void_p(triangles.data_ptr()), n, ctypes.byref(cs),
            ctypes.c_void_p(out_nodes.data_ptr()), cap, ctypes.byref(count), lens_p,
            ctypes.c_void_p(out_perm.data_ptr()), ctypes.byref(st))
    else:
        n = aabbs.shape[0]
        rc = L.mgbvh_build_aabbs_dev(
            ctx.ptr, ctypes.c_void_p(aabbs.data_ptr()), n, ctypes.byref(cs),
            ctypes.c_void_p(out_nodes.data_ptr()), cap, ctypes.byref(count), lens_p,
            ctypes.c_void_p(out_perm.data_ptr()), ctypes.byref(st))
    ctx.check(rc)
    return count.value, rc, st.as_dict()


def build_batch_device(ctx: Context, settings: BvhSettings, meshes, out_nodes, out_perm, *,
                       out_lens=None, min_leaf_objects: int = 1, max_leaf_objects: int = 1,
                       stream=None):
    """Batched build: one BVH per mesh (BLAS per mesh, the TLAS as one more
    mesh of instance AABBs), all in one pass.

    meshes: list of dicts, each either {"vertices": float32 [V, k] tensor,
    "triangles": int32 [N, 3] tensor} or {"aabbs": float32 [N, 6] tensor},
    plus optional "bounds" (6 floats; BvhSettings::bounds of that mesh).
    Returns (node_offsets [len(meshes) + 1], status, stats): mesh m's nodes
    are out_nodes rows node_offsets[m]..node_offsets[m+1] (child links local
    to that range), its permutation is out_perm[first:first + N_m].
    """
    import torch

    L = ctx.L
    s = stream if stream is not None else torch.cuda.current_stream()
    ctx.set_stream(s.cuda_stream)
    cs = settings.to_c(min_leaf_objects, max_leaf_objects)
    descs = (_lib.MeshDesc * max(len(meshes), 1))()
    for i, m in enumerate(meshes):
        d = descs[i]
        if "aabbs" in m:
            d.aabbs = m["aabbs"].data_ptr()
            d.count = m["aabbs"].shape[0]
        else:
            d.vertices = m["vertices"].data_ptr()
            d.vertex_stride_bytes = m["vertices"].shape[1] * 4
            d.vertex_count = m["vertices"].shape[0]
            d.triangles = m["triangles"].data_ptr()
            d.count = m["triangles"].shape[0]
        if m.get("bounds") is not None:
            d.has_bounds = 1
            for k in range(6):
                d.bounds[k] = float(m["bounds"][k])
    offs = (ctypes.c_uint32 * (len(meshes) + 1))()
    st = _lib.Stats()
    cap = out_nodes.numel() * out_nodes.element_size() // 32
    rc = L.mgbvh_build_batch_dev(ctx.ptr, descs, len(meshes), ctypes.byref(cs),
                                 ctypes.c_void_p(out_nodes.data_ptr()), cap,
                                 ctypes.c_void_p(out_lens.data_ptr()) if out_lens is not None else None,
                                 ctypes.c_void_p(out_perm.data_ptr()), offs, ctypes.byref(st))
    ctx.check(rc)
    return list(offs), rc, st.as_dict()


def instance_aabbs_device(ctx: Context, mesh_bounds, instance_mesh, transforms, out_aabbs) -> None:
    """World AABBs of instances on the GPU (the TLAS input of marigold's scene
    upload, marigold/src/app/data/scene/model.rs:191-234). Device tensors:
    mesh_bounds float32 [M, 6], instance_mesh int32/uint32 [I], transforms
    float32 [I, 16] (column-major), out_aabbs float32 [I, 6]. Runs on the
    context's stream; raises MgbvhError for an index past M."""
    n = instance_mesh.shape[0]
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    ctx.check(ctx.L.mgbvh_instance_aabbs_dev(ctx.ptr, vp(mesh_bounds), mesh_bounds.shape[0],
                                             vp(instance_mesh), vp(transforms), n, vp(out_aabbs)))


class Scene:
    """A two-level scene on the device, laid out as marigold uploads it for its
    scene shader (marigold/src/app/data/scene/model.rs:167-234,
    geometry/mod.rs:175-199): the TLAS nodes, the instance records in the TLAS
    build's permuted order (inverse transform + mesh index), the mesh table
    (BLAS root, triangle offset and count, vertex offset), the BLAS nodes of
    every mesh, the vertex positions and every mesh's triangles in its BLAS
    build's permuted order, vertex indices relative to the mesh's vertex
    offset.

    from_batch assembles it from one batched build (build_batch_device) whose
    descriptors were the meshes followed by the TLAS over the instances' world
    boxes: `meshes` the (vertices [V, k], triangles [N, 3]) device tensors of
    the BLAS meshes, `offsets`, `nodes`, `lens`, `perm` that build's outputs,
    `instance_mesh` [I] and `transforms` [I, 16] (column-major, mesh ->
    world) the instances in their original order. The inverse transforms are
    computed in float64 and rounded to float32."""

    def __init__(self, **tensors):
        self.__dict__.update(tensors)

    @classmethod
    def from_batch(cls, meshes, offsets, nodes, lens, perm, instance_mesh, transforms):
        import torch
        m = len(meshes)
        dev = nodes.device
        counts = [int(t.shape[0]) for _, t in meshes]
        tri_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        vcounts = [int(v.shape[0]) for v, _ in meshes]
        v_off = np.concatenate([[0], np.cumsum(vcounts)]).astype(np.int64)
        tris, verts = [], []
        for k, (v, t) in enumerate(meshes):
            p = perm[tri_off[k]:tri_off[k + 1]].long()
            tris.append(t.reshape(-1, 3)[p].to(torch.int32))
            verts.append(v[:, :3].float())
        mesh_tab = torch.tensor(np.stack([np.asarray(offsets[:m], np.int64), tri_off[:m],
                                          np.asarray(counts, np.int64), v_off[:m]], 1).astype(np.uint32).view(np.int32),
                                device=dev)
        n_inst = int(instance_mesh.shape[0])
        tlas_first = int(tri_off[m])
        tlas_perm = perm[tlas_first:tlas_first + n_inst].long()
        a = transforms.double().reshape(-1, 4, 4).transpose(1, 2)  # [instance, row, column]
        inv = torch.linalg.inv(a).transpose(1, 2).reshape(-1, 16).float()  # back to column-major
        rec = torch.zeros((n_inst, 20), dtype=torch.int32, device=dev)
        rec[:, :16] = inv.view(torch.int32)
        rec[:, 16] = instance_mesh.to(torch.int32)
        rec = rec[tlas_perm].contiguous()
        lo, hi = int(offsets[m]), int(offsets[m + 1])
        return cls(tlas_nodes=nodes[lo * 8:hi * 8], tlas_count=hi - lo,
                   tlas_lens=None if lens is None else lens[lo:hi],
                   instances=rec, instance_count=n_inst, meshes=mesh_tab, mesh_count=m,
                   blas_nodes=nodes[:lo * 8], blas_count=lo, blas_lens=None if lens is None else lens[:lo],
                   vertices=torch.cat(verts).contiguous(), triangles=torch.cat(tris).contiguous(),
                   triangle_count=int(tri_off[m]), instance_order=tlas_perm)

    def bind(self, tracer, stream=None):
        """mgbvh_tracer_set_scene_dev on `tracer` (an _lib.Tracer)."""
        vp = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        tracer.check(tracer.L.mgbvh_tracer_set_scene_dev(
            tracer.ptr, vp(self.tlas_nodes), self.tlas_count, vp(self.tlas_lens), vp(self.instances),
            self.instance_count, vp(self.meshes), self.mesh_count, vp(self.blas_nodes), self.blas_count,
            vp(self.blas_lens), vp(self.vertices), 12, int(self.vertices.shape[0]), vp(self.triangles),
            self.triangle_count, sp))


def trace_scene_device(tracer, rays, *, stream=None, bruteforce=False, cull=False):
    """Closest hits of rays (float32 [n, 8] device tensor) through the scene
    bound to `tracer`: (t float32 [n], instance int32 [n], triangle int32 [n],
    counters or None, device seconds or None). bruteforce=True runs the
    brute-force check instead of the traversal."""
    import torch
    n = int(rays.shape[0])
    t = torch.empty(n, dtype=torch.float32, device=rays.device)
    hi = torch.empty(n, dtype=torch.int32, device=rays.device)
    hp = torch.empty(n, dtype=torch.int32, device=rays.device)
    vp = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    if bruteforce:
        tracer.check(tracer.L.mgbvh_trace_scene_bruteforce_dev(tracer.ptr, vp(rays), n, vp(t), vp(hi), vp(hp),
                                                               1 if cull else 0, sp))
        return t, hi, hp, None, None
    counts = (ctypes.c_uint64 * 3)()
    secs = ctypes.c_double(0)
    tracer.check(tracer.L.mgbvh_trace_scene_dev(tracer.ptr, vp(rays), n, vp(t), vp(hi), vp(hp), counts,
                                                ctypes.byref(secs), sp))
    return t, hi, hp, list(counts), secs.value
