"""Writes small glTF 2.0 scenes for the loader tests (no meshes ship with the
reference): a .gltf with an external .bin, the same scene as a .glb, or with
the buffer as a data: URI."""
from __future__ import annotations

import base64
import json
import os
import struct

import numpy as np


class _Buf:
    def __init__(self):
        self.data = bytearray()
        self.views, self.accessors = [], []

    def view(self, arr: np.ndarray, stride: int = 0) -> int:
        while len(self.data) % 4:
            self.data.append(0)
        v = {"buffer": 0, "byteOffset": len(self.data), "byteLength": arr.nbytes}
        if stride:
            v["byteStride"] = stride
        self.data += arr.tobytes()
        self.views.append(v)
        return len(self.views) - 1

    def accessor(self, view: int, ctype: int, count: int, kind: str, offset: int = 0, **extra) -> int:
        a = {"bufferView": view, "componentType": ctype, "count": count, "type": kind}
        if offset:
            a["byteOffset"] = offset
        a.update(extra)
        self.accessors.append(a)
        return len(self.accessors) - 1


def mesh_primitive(buf: _Buf, vertices: np.ndarray, triangles: np.ndarray, *, uv_u8: bool = False,
                   interleaved: bool = False, index_type: int = 5125, extra_indices: int = 0) -> dict:
    """A triangle primitive from vertex records [V, 8] (pos, uv.x, normal,
    uv.y) and index triples; the POSITION accessor carries min/max."""
    pos = np.ascontiguousarray(vertices[:, 0:3], np.float32)
    nrm = np.ascontiguousarray(vertices[:, 4:7], np.float32)
    uv = np.ascontiguousarray(vertices[:, [3, 7]], np.float32)
    n = pos.shape[0]
    mn, mx = pos.min(axis=0).tolist(), pos.max(axis=0).tolist()
    if interleaved:
        rec = np.zeros((n, 8), np.float32)
        rec[:, 0:3], rec[:, 3:6], rec[:, 6:8] = pos, nrm, uv
        v = buf.view(rec, stride=32)
        ap = buf.accessor(v, 5126, n, "VEC3", min=mn, max=mx)
        an = buf.accessor(v, 5126, n, "VEC3", offset=12)
        at = buf.accessor(v, 5126, n, "VEC2", offset=24)
    else:
        ap = buf.accessor(buf.view(pos), 5126, n, "VEC3", min=mn, max=mx)
        an = buf.accessor(buf.view(nrm), 5126, n, "VEC3")
        if uv_u8:
            at = buf.accessor(buf.view(np.round(uv * 255).astype(np.uint8)), 5121, n, "VEC2", normalized=True)
        else:
            at = buf.accessor(buf.view(uv), 5126, n, "VEC2")
    flat = np.concatenate([triangles.reshape(-1), np.zeros(extra_indices, np.uint32)])
    dt = {5121: np.uint8, 5123: np.uint16, 5125: np.uint32}[index_type]
    ai = buf.accessor(buf.view(flat.astype(dt)), index_type, flat.shape[0], "SCALAR")
    return {"attributes": {"POSITION": ap, "NORMAL": an, "TEXCOORD_0": at}, "indices": ai}


def write(path: str, doc: dict, buf: _Buf, form: str) -> str:
    """form: 'gltf' (.gltf + .bin in directory `path`), 'glb' (file
    path/scene.glb) or 'data' (.gltf with a data: URI buffer)."""
    os.makedirs(path, exist_ok=True)
    doc = dict(doc)
    doc["asset"] = {"version": "2.0"}
    doc["bufferViews"], doc["accessors"] = buf.views, buf.accessors
    data = bytes(buf.data)
    if form == "gltf":
        doc["buffers"] = [{"uri": "scene.bin", "byteLength": len(data)}]
        with open(os.path.join(path, "scene.bin"), "wb") as fh:
            fh.write(data)
        out = os.path.join(path, "scene.gltf")
        with open(out, "w") as fh:
            json.dump(doc, fh)
        return path
    if form == "data":
        doc["buffers"] = [{"uri": "data:application/octet-stream;base64," + base64.b64encode(data).decode(),
                           "byteLength": len(data)}]
        out = os.path.join(path, "scene.gltf")
        with open(out, "w") as fh:
            json.dump(doc, fh)
        return out
    doc["buffers"] = [{"byteLength": len(data)}]
    js = json.dumps(doc).encode()
    js += b" " * (-len(js) % 4)
    binc = data + b"\0" * (-len(data) % 4)
    total = 12 + 8 + len(js) + 8 + len(binc)
    out = os.path.join(path, "scene.glb")
    with open(out, "wb") as fh:
        fh.write(struct.pack("<III", 0x46546C67, 2, total))
        fh.write(struct.pack("<II", len(js), 0x4E4F534A) + js)
        fh.write(struct.pack("<II", len(binc), 0x004E4942) + binc)
    return out


def buffer() -> _Buf:
    return _Buf()
