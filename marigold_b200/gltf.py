"""glTF 2.0 scenes into the builder's inputs.

Host side of the reference's loader (gltf_loading/src/lib.rs:26-187, on the
`gltf` crate 1.4): every triangle-mode mesh primitive becomes a mesh of
32-byte vertex records (position, uv.x, normal, uv.y; the reference's
MeshVertex), index triples and the POSITION accessor's bounds, and every scene
becomes a list of instances (the node's global transform and the mesh it
draws). `to_device` puts the meshes in device tensors in the form
`build_batch_device` takes, so a scene's BLASes build in one batched pass and
its TLAS from the instance boxes `instance_aabbs_device` computes.

Formats read: a directory holding a `.gltf` file (the reference's
convention), a `.gltf` file, or a `.glb` file; buffers from files next to the
`.gltf`, `data:` URIs or the GLB binary chunk; accessors of any component
type with or without a byte stride. Sparse accessors are rejected.

Differences from the reference, on purpose: meshes are numbered in
(mesh, primitive) order (the reference numbers them in the iteration order of
a hash map, which varies between runs), and a node's TRS transform is
composed as T * R * S in f32 by the glTF specification's formulas (matrix
nodes are taken as written).
"""
from __future__ import annotations

import base64
import json
import logging
import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

log = logging.getLogger("marigold_b200.gltf")

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32,
              5126: np.float32}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}
_MODE_TRIANGLES = 4
_GLB_MAGIC, _CHUNK_JSON, _CHUNK_BIN = 0x46546C67, 0x4E4F534A, 0x004E4942
_F = np.float32


@dataclass
class Mesh:
    """UnserializedMesh (mesh_interface/src/lib.rs:34-38)."""
    vertices: np.ndarray   # float32 [V, 8]: position xyz, uv.x, normal xyz, uv.y
    triangles: np.ndarray  # uint32 [N, 3]
    bounds: np.ndarray     # float32 [6]: the POSITION accessor's min xyz, max xyz


@dataclass
class Instance:
    """MeshInstance (mesh_interface/src/lib.rs:45-48)."""
    transform: np.ndarray  # float32 [16], column-major (glam Mat4 layout)
    mesh_index: object     # (mesh, primitive) in GltfScenes, a packed index after into_meshes_and_scenes


@dataclass
class Scene:
    name: str
    instances: List[Instance] = field(default_factory=list)


# ------------------------------------------------------------------ f32 matrix algebra (glam order)

def mat4_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a * b for column-major f32 4x4 matrices ([16] each): column j of the
    product is ((a.c0 * b[j].x + a.c1 * b[j].y) + a.c2 * b[j].z) + a.c3 * b[j].w,
    every product and sum rounded to f32 (glam's Mat4 * Mat4)."""
    A = np.asarray(a, _F).reshape(4, 4)  # [column, row]
    B = np.asarray(b, _F).reshape(4, 4)
    out = np.empty((4, 4), _F)
    for j in range(4):
        acc = A[0] * B[j, 0]
        acc = (acc + A[1] * B[j, 1]).astype(_F)
        acc = (acc + A[2] * B[j, 2]).astype(_F)
        acc = (acc + A[3] * B[j, 3]).astype(_F)
        out[j] = acc
    return out.reshape(16)


def trs_matrix(translation, rotation, scale) -> np.ndarray:
    """T * R * S (glTF node transform) in f32; rotation is a unit quaternion
    (x, y, z, w)."""
    x, y, z, w = (_F(v) for v in rotation)
    two = _F(2.0)
    xx, yy, zz = x * x * two, y * y * two, z * z * two
    xy, xz, yz = x * y * two, x * z * two, y * z * two
    wx, wy, wz = w * x * two, w * y * two, w * z * two
    one = _F(1.0)
    r = np.array([[one - yy - zz, xy + wz, xz - wy, 0],      # column 0
                  [xy - wz, one - xx - zz, yz + wx, 0],      # column 1
                  [xz + wy, yz - wx, one - xx - yy, 0],      # column 2
                  [0, 0, 0, one]], _F)
    s = np.diag(np.array([scale[0], scale[1], scale[2], 1.0], _F)).astype(_F)
    t = np.eye(4, dtype=_F)
    t[3, 0:3] = np.asarray(translation, _F)
    return mat4_mul(mat4_mul(t.reshape(16), r.reshape(16)), s.reshape(16))


def _node_matrix(node: dict) -> np.ndarray:
    if "matrix" in node:
        return np.asarray(node["matrix"], _F)
    return trs_matrix(node.get("translation", [0.0, 0.0, 0.0]), node.get("rotation", [0.0, 0.0, 0.0, 1.0]),
                      node.get("scale", [1.0, 1.0, 1.0]))


def _uniform_scale(m: np.ndarray) -> bool:
    """Mat4::to_scale_rotation_translation's scale: the column lengths, the
    first negated for a negative determinant; True when all three agree."""
    c = np.asarray(m, np.float64).reshape(4, 4)[:3, :3]
    s = np.sqrt((c * c).sum(axis=1)).astype(_F)
    if np.linalg.det(c) < 0:
        s[0] = -s[0]
    return bool(s[0] == s[1] == s[2])


# ------------------------------------------------------------------ file and buffer access

def _read_document(path: str) -> Tuple[dict, str, Optional[bytes]]:
    if os.path.isdir(path):
        # the reference's convention: the directory holds the .gltf and its assets
        names = sorted(f for f in os.listdir(path) if f.endswith(".gltf"))
        if not names:
            raise FileNotFoundError(f"gltf path {path} wasn't valid")
        path = os.path.join(path, names[0])
    base = os.path.dirname(os.path.abspath(path))
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) >= 12 and struct.unpack_from("<I", data, 0)[0] == _GLB_MAGIC:
        version, length = struct.unpack_from("<II", data, 4)
        if version != 2:
            raise ValueError(f"{path}: GLB version {version} (2 expected)")
        doc, blob, off = None, None, 12
        while off + 8 <= min(length, len(data)):
            clen, ctype = struct.unpack_from("<II", data, off)
            chunk = data[off + 8: off + 8 + clen]
            if ctype == _CHUNK_JSON and doc is None:
                doc = json.loads(chunk.decode("utf-8"))
            elif ctype == _CHUNK_BIN and blob is None:
                blob = bytes(chunk)
            off += 8 + clen
        if doc is None:
            raise ValueError(f"{path}: GLB without a JSON chunk")
        return doc, base, blob
    return json.loads(data.decode("utf-8")), base, None


def _load_buffers(doc: dict, base: str, blob: Optional[bytes]) -> List[bytes]:
    out = []
    for i, b in enumerate(doc.get("buffers", [])):
        uri = b.get("uri")
        if uri is None:
            if blob is None:
                raise ValueError(f"buffer {i} has no uri and there is no GLB binary chunk")
            data = blob
        elif uri.startswith("data:"):
            data = base64.b64decode(uri.split(",", 1)[1])
        else:
            with open(os.path.join(base, uri), "rb") as fh:
                data = fh.read()
        if len(data) < b.get("byteLength", 0):
            raise ValueError(f"buffer {i} holds {len(data)} bytes, byteLength is {b['byteLength']}")
        out.append(data)
    return out


def read_accessor(doc: dict, buffers: List[bytes], index: int) -> np.ndarray:
    """Accessor `index` as an array [count, components] of its component type."""
    acc = doc["accessors"][index]
    if "sparse" in acc:
        raise ValueError(f"accessor {index}: sparse accessors are not supported")
    dtype = np.dtype(_COMPONENT[acc["componentType"]])
    nc = _NCOMP[acc["type"]]
    count = acc["count"]
    if "bufferView" not in acc:
        return np.zeros((count, nc), dtype)
    view = doc["bufferViews"][acc["bufferView"]]
    data = buffers[view["buffer"]]
    start = view.get("byteOffset", 0) + acc.get("byteOffset", 0)
    elem = dtype.itemsize * nc
    stride = view.get("byteStride", elem) or elem
    if count and start + stride * (count - 1) + elem > view.get("byteOffset", 0) + view["byteLength"]:
        raise ValueError(f"accessor {index} reads past its buffer view")
    arr = np.ndarray((count, nc), dtype, buffer=data, offset=start, strides=(stride, dtype.itemsize))
    return np.array(arr)  # a compact copy


def _texcoords_f32(a: np.ndarray) -> np.ndarray:
    """ReadTexCoords::into_f32: unsigned normalized bytes and shorts divided
    by 255 and 65535 in f32, floats as they are."""
    if a.dtype == np.uint8:
        return (a.astype(_F) / _F(255.0)).astype(_F)
    if a.dtype == np.uint16:
        return (a.astype(_F) / _F(65535.0)).astype(_F)
    if a.dtype == np.float32:
        return a
    raise ValueError(f"TEXCOORD_0 of component type {a.dtype} is not readable as f32")


# ------------------------------------------------------------------ scenes

class GltfScenes:
    """GltfScenes (gltf_loading/src/lib.rs:20-23): meshes keyed by
    (mesh, primitive) and the scenes' instances."""

    def __init__(self, meshes: Dict[Tuple[int, int], Mesh], scenes: List[Scene]):
        self.meshes = meshes
        self.scenes = scenes

    @classmethod
    def load(cls, path: str) -> "GltfScenes":
        """GltfScenes::load (lib.rs:56-187)."""
        doc, base, blob = _read_document(str(path))
        buffers = _load_buffers(doc, base, blob)
        meshes: Dict[Tuple[int, int], Mesh] = {}
        for mi, mesh in enumerate(doc.get("meshes", [])):
            for pi, prim in enumerate(mesh.get("primitives", [])):
                if prim.get("mode", _MODE_TRIANGLES) != _MODE_TRIANGLES:
                    continue
                meshes[(mi, pi)] = _read_primitive(doc, buffers, prim, (mi, pi))
        scenes = []
        nodes = doc.get("nodes", [])
        for si, sc in enumerate(doc.get("scenes", [])):
            scene = Scene(sc.get("name", f"unnamed scene #{si}"))
            for n in sc.get("nodes", []):
                _traverse(doc, nodes, n, np.eye(4, dtype=_F).reshape(16), scene.instances, 0)
            scenes.append(scene)
        for key, m in sorted(meshes.items()):
            log.info("Mesh #%s of mesh at path %s has %d vertices and %d triangles", key, path,
                     m.vertices.shape[0], m.triangles.shape[0])
        log.info("Creating %d scenes (%d unique meshes)", len(scenes), len(meshes))
        return cls(meshes, scenes)

    def into_meshes_and_scenes(self) -> Tuple[List[Mesh], List[Scene]]:
        """GltfScenes::into_meshes_and_scenes (lib.rs:189-221), meshes packed
        in (mesh, primitive) order."""
        keys = sorted(self.meshes)
        packed = {k: i for i, k in enumerate(keys)}
        scenes = [Scene(s.name, [Instance(i.transform, packed[i.mesh_index]) for i in s.instances])
                  for s in self.scenes]
        return [self.meshes[k] for k in keys], scenes


def _read_primitive(doc, buffers, prim, key) -> Mesh:
    attrs = prim.get("attributes", {})
    for name in ("POSITION", "NORMAL", "TEXCOORD_0"):
        if name not in attrs:
            what = {"POSITION": "positions", "NORMAL": "normals", "TEXCOORD_0": "uvs from TEXCOORD_0"}[name]
            raise ValueError(f"mesh {key}: couldn't read mesh {what}")
    if "indices" not in prim:
        raise ValueError(f"mesh {key}: couldn't read mesh indices")
    pos = read_accessor(doc, buffers, attrs["POSITION"])
    nrm = read_accessor(doc, buffers, attrs["NORMAL"])
    uv = _texcoords_f32(read_accessor(doc, buffers, attrs["TEXCOORD_0"]))
    if pos.dtype != np.float32 or pos.shape[1] != 3 or nrm.dtype != np.float32 or nrm.shape[1] != 3:
        raise ValueError(f"mesh {key}: POSITION and NORMAL must be float VEC3")
    # the reference zips the three streams: the shortest one sets the count
    nv = min(pos.shape[0], nrm.shape[0], uv.shape[0])
    v = np.empty((nv, 8), _F)
    v[:, 0:3] = pos[:nv]
    v[:, 3] = uv[:nv, 0]
    v[:, 4:7] = nrm[:nv]
    v[:, 7] = uv[:nv, 1]
    idx = read_accessor(doc, buffers, prim["indices"])
    if idx.dtype not in (np.uint8, np.uint16, np.uint32) or idx.shape[1] != 1:
        raise ValueError(f"mesh {key}: indices must be unsigned SCALAR")
    flat = idx[:, 0].astype(np.uint32)
    tris = flat[: (flat.shape[0] // 3) * 3].reshape(-1, 3)  # array_chunks::<3> drops a remainder
    pacc = doc["accessors"][attrs["POSITION"]]
    if "min" not in pacc or "max" not in pacc:
        raise ValueError(f"mesh {key}: the POSITION accessor has no min/max (the primitive's bounding box)")
    bounds = np.array(list(pacc["min"]) + list(pacc["max"]), _F)
    return Mesh(v, np.ascontiguousarray(tris), bounds)


def _traverse(doc, nodes, index, parent, out: List[Instance], depth: int) -> None:
    """GltfScenes::traverse_scene (lib.rs:26-54)."""
    if depth > len(nodes):
        raise ValueError("the node hierarchy has a cycle")
    node = nodes[index]
    local = _node_matrix(node)
    if not _uniform_scale(local):
        log.warning("Encountered a non-uniform scale in a gltf transform")
    glob = mat4_mul(parent, local)
    if "mesh" in node:
        mesh = doc["meshes"][node["mesh"]]
        for pi, prim in enumerate(mesh.get("primitives", [])):
            if prim.get("mode", _MODE_TRIANGLES) == _MODE_TRIANGLES:
                out.append(Instance(glob.copy(), (node["mesh"], pi)))
    for c in node.get("children", []):
        _traverse(doc, nodes, c, glob, out, depth + 1)


# ------------------------------------------------------------------ device buffers

def to_device(meshes: List[Mesh], device: str = "cuda") -> List[dict]:
    """The meshes as device tensors in `build_batch_device`'s form (vertex
    records float32 [V, 8], triangles int32 [N, 3], the accessor bounds as
    the mesh's root bounds, as the reference passes them, model.rs:83)."""
    import torch
    return [{"vertices": torch.from_numpy(m.vertices).to(device),
             "triangles": torch.from_numpy(m.triangles.view(np.int32)).to(device),
             "bounds": [float(x) for x in m.bounds]} for m in meshes]


def instance_arrays(scene: Scene) -> Tuple[np.ndarray, np.ndarray]:
    """A packed scene's instances as (mesh index uint32 [I], transforms
    float32 [I, 16]) for `instance_aabbs_device` / `synth.instance_aabbs`."""
    ids = np.array([i.mesh_index for i in scene.instances], np.uint32)
    tf = np.stack([i.transform for i in scene.instances]).astype(_F) if scene.instances else np.zeros((0, 16), _F)
    return ids, tf
