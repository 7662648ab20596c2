"""Seeded synthetic inputs for the builder: meshes, scenes and rays.

Every generator is counter based (one hash per element, no sequential RNG
state), so any slice of a workload can be regenerated on its own and the
same seed gives the same f32 data on every host. Only IEEE-exact float64
operations are used (add, multiply, divide, sqrt, floor); sine and cosine are
evaluated by a fixed Taylor polynomial, so no platform libm enters the data.
Negative zeros are canonicalised to +0.0, as the builder's min/max semantics
leave the sign of a zero unspecified. (The mixed scene's Gaussian blobs use
numpy's log for the Box-Muller transform; its data is generated where it is
used and never pinned by a committed hash.)

Vertices use marigold's 32-byte MeshVertex layout (position xyz, uv_x,
normal xyz, uv_y; mesh_interface/src/lib.rs:6-12) with zero normals and uvs.
Triangles are MeshTriangle index triples (mesh_interface/src/lib.rs:14-17).
"""
from __future__ import annotations

import numpy as np

_M32 = np.uint64(0xFFFFFFFF)


def pcg_hash(v):
    """PCG-RXS-M-XS 32-bit hash (O'Neill's PCG output permutation applied to
    one LCG step, as popularised by Jarzynski & Olano 2020). uint32 in/out."""
    v = np.asarray(v, dtype=np.uint32)
    with np.errstate(over="ignore"):
        state = v * np.uint32(747796405) + np.uint32(2891336453)
        word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
    return (word >> np.uint32(22)) ^ word


def stream_key(seed: int, stream: int) -> np.uint32:
    s = pcg_hash(np.uint32(seed & 0xFFFFFFFF))
    with np.errstate(over="ignore"):
        return pcg_hash(s ^ pcg_hash(np.uint32(stream & 0xFFFFFFFF) + np.uint32(0x9E3779B9)))


def uniform(seed: int, stream: int, idx) -> np.ndarray:
    """float64 uniform in [0, 1) with 24 random bits, element idx of a stream."""
    k = stream_key(seed, stream)
    with np.errstate(over="ignore"):
        h = pcg_hash(np.asarray(idx, dtype=np.uint32) + k)
    return (h >> np.uint32(8)).astype(np.float64) * (1.0 / 16777216.0)


def _sincos(x):
    """sin and cos of x in [-pi, pi] by a fixed Taylor polynomial (|err| < 1e-15)."""
    x = np.asarray(x, dtype=np.float64)
    x2 = x * x
    term_s = x.copy()
    term_c = np.ones_like(x)
    s = term_s.copy()
    c = term_c.copy()
    for k in range(1, 16):
        term_s = term_s * x2 / ((2 * k) * (2 * k + 1)) * -1.0
        term_c = term_c * x2 / ((2 * k - 1) * (2 * k)) * -1.0
        s = s + term_s
        c = c + term_c
    return s, c


def unit_vectors(seed: int, stream: int, idx) -> np.ndarray:
    """Directions uniform on the sphere: z = 2u - 1, phi = 2 pi v."""
    z = 2.0 * uniform(seed, stream, idx) - 1.0
    phi = (2.0 * uniform(seed, stream + 1, idx) - 1.0) * np.pi
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    s, c = _sincos(phi)
    return np.stack([r * c, r * s, z], axis=-1)


def _f32(a) -> np.ndarray:
    out = np.asarray(a, dtype=np.float32)
    return out + np.float32(0.0)  # -0.0 -> +0.0


def pack_vertices(pos: np.ndarray) -> np.ndarray:
    """float32 [V, 8] MeshVertex records with the given positions."""
    v = np.zeros((pos.shape[0], 8), dtype=np.float32)
    v[:, 0:3] = _f32(pos)
    return v


def mesh_bounds(vertices: np.ndarray) -> np.ndarray:
    """Accessor-style bounds (min xyz, max xyz) over the vertex positions."""
    p = vertices[:, 0:3]
    return np.concatenate([p.min(axis=0), p.max(axis=0)]).astype(np.float32)


def triangle_aabbs(vertices: np.ndarray, triangles: np.ndarray) -> np.ndarray:
    """float32 [N, 6] AABBs (MeshTriangle::bounding_volume)."""
    p = vertices[:, 0:3][triangles]  # [N, 3, 3]
    return np.concatenate([p.min(axis=1), p.max(axis=1)], axis=1).astype(np.float32)


def random_triangles(n: int, seed: int = 1):
    """Small random triangles: vertex 0 uniform in [0,1]^3, vertices 1 and 2
    offset from it by lengths U(0.001, 0.02) in uniform directions. Vertices
    are not shared: triangle i uses vertices 3i, 3i+1, 3i+2."""
    i = np.arange(n, dtype=np.uint32)
    v0 = np.stack([uniform(seed, s, i) for s in (0, 1, 2)], axis=-1)
    pts = [v0]
    for k in (1, 2):
        length = 0.001 + 0.019 * uniform(seed, 10 * k, i)
        d = unit_vectors(seed, 10 * k + 1, i)
        pts.append(v0 + length[:, None] * d)
    pos = np.stack(pts, axis=1).reshape(3 * n, 3)
    vertices = pack_vertices(pos)
    triangles = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return vertices, triangles


_PHI = (1.0 + np.sqrt(5.0)) / 2.0
_ICO_V = np.array([
    [-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
    [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
    [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1]], dtype=np.float64)
_ICO_F = np.array([
    [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
    [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
    [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
    [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)


def _normalize(p):
    return p / np.sqrt((p * p).sum(axis=1, keepdims=True))


def icosphere(level: int):
    """Unit icosphere subdivided `level` times: 20*4^L faces, 10*4^L+2 vertices."""
    v = _normalize(_ICO_V.copy())
    f = _ICO_F.copy()
    for _ in range(level):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        key = np.minimum(e[:, 0], e[:, 1]) * nv + np.maximum(e[:, 0], e[:, 1])
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // nv
        b = uniq % nv
        mid = _normalize((v[a] + v[b]) * 0.5)
        m = inv.reshape(3, -1) + nv  # midpoint ids of edges (01, 12, 20)
        m01, m12, m20 = m[0], m[1], m[2]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], axis=1),
            np.stack([f[:, 1], m12, m01], axis=1),
            np.stack([f[:, 2], m20, m12], axis=1),
            np.stack([m01, m12, m20], axis=1)], axis=0)
        v = np.concatenate([v, mid], axis=0)
    return v, f


def _lattice(seed: int, octave: int, ix, iy, iz):
    k = stream_key(seed, 1000 + octave)
    with np.errstate(over="ignore"):
        h = pcg_hash((ix.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32) ^ k)
        h = pcg_hash(h ^ (iy.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32))
        h = pcg_hash(h ^ (iz.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32))
    return (h >> np.uint32(8)).astype(np.float64) * (2.0 / 16777216.0) - 1.0


def value_noise(p: np.ndarray, seed: int, octaves=(1.0, 2.0, 4.0), amps=(1.0, 0.5, 0.25)):
    """3-octave value noise on a hashed integer lattice, smoothstep-weighted
    trilinear interpolation, normalised by the amplitude sum (range [-1, 1])."""
    total = np.zeros(p.shape[0], dtype=np.float64)
    for o, (freq, amp) in enumerate(zip(octaves, amps)):
        q = p * freq
        q0 = np.floor(q)
        t = q - q0
        w = t * t * (3.0 - 2.0 * t)
        i0 = q0.astype(np.int64)
        acc = np.zeros(p.shape[0], dtype=np.float64)
        for dx in (0, 1):
            wx = w[:, 0] if dx else 1.0 - w[:, 0]
            for dy in (0, 1):
                wy = w[:, 1] if dy else 1.0 - w[:, 1]
                for dz in (0, 1):
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    val = _lattice(seed, o, i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
                    acc = acc + val * (wx * wy * wz)
        total = total + amp * acc
    return total / float(sum(amps))


def noisy_icosphere(level: int = 8, seed: int = 2, amplitude: float = 0.05):
    """Icosphere with vertices displaced radially by 1 + amplitude * noise(p)."""
    v, f = icosphere(level)
    r = 1.0 + amplitude * value_noise(v, seed)
    vertices = pack_vertices(v * r[:, None])
    return vertices, f.astype(np.uint32)


def config1_mesh(seed: int = 1):
    """65,536 random small triangles (the binned-SAH BLAS workload)."""
    return random_triangles(65536, seed)


def config2_mesh(seed: int = 2):
    """Noisy icosphere, level 8: 1,310,720 triangles, 655,362 shared vertices."""
    return noisy_icosphere(8, seed)


def gaussian(seed: int, stream: int, idx) -> np.ndarray:
    """Standard normal samples by the Box-Muller transform of two uniforms."""
    u1 = uniform(seed, stream, idx)
    u2 = uniform(seed, stream + 1, idx)
    r = np.sqrt(-2.0 * np.log(1.0 - u1))
    s, c = _sincos((2.0 * u2 - 1.0) * np.pi)
    return r * c


def mixed_scene(seed: int = 5, blobs: int = 64, n_blob: int = 8388608, grid=(2048, 1024),
                n_thin: int = 4194304):
    """The large mixed scene: n_blob small triangles in `blobs` Gaussian blobs
    (sigma uniform in [0.5, 5]), a flat ground grid of grid[0] x grid[1] quads
    split into two triangles each, and n_thin long thin triangles (aspect
    1:200, random orientation). Vertices are unshared and stored compactly as
    float32 [3N, 3] (12-byte stride); triangles are [3i, 3i+1, 3i+2]."""
    parts = []
    # blobs
    b = np.arange(blobs, dtype=np.uint32)
    centers = np.stack([uniform(seed, 1, b) * 160.0 - 80.0, uniform(seed, 2, b) * 60.0,
                        uniform(seed, 3, b) * 160.0 - 80.0], axis=-1)
    sigma = 0.5 + 4.5 * uniform(seed, 4, b)
    i = np.arange(n_blob, dtype=np.uint32)
    which = (i % blobs).astype(np.int64)
    v0 = centers[which] + sigma[which, None] * np.stack(
        [gaussian(seed, 10 + 2 * k, i) for k in range(3)], axis=-1)
    e1 = unit_vectors(seed, 20, i) * (0.02 + 0.18 * uniform(seed, 22, i))[:, None]
    e2 = unit_vectors(seed, 23, i) * (0.02 + 0.18 * uniform(seed, 25, i))[:, None]
    parts.append(np.stack([v0, v0 + e1, v0 + e2], axis=1))
    # ground grid on y = 0 over [-100, 100]^2
    gx, gz = grid
    xs = np.linspace(-100.0, 100.0, gx + 1)
    zs = np.linspace(-100.0, 100.0, gz + 1)
    qx, qz = np.meshgrid(np.arange(gx), np.arange(gz), indexing="ij")
    qx = qx.ravel()
    qz = qz.ravel()
    p00 = np.stack([xs[qx], np.zeros(qx.size), zs[qz]], axis=-1)
    p10 = np.stack([xs[qx + 1], np.zeros(qx.size), zs[qz]], axis=-1)
    p01 = np.stack([xs[qx], np.zeros(qx.size), zs[qz + 1]], axis=-1)
    p11 = np.stack([xs[qx + 1], np.zeros(qx.size), zs[qz + 1]], axis=-1)
    t_a = np.stack([p00, p10, p11], axis=1)
    t_b = np.stack([p00, p11, p01], axis=1)
    parts.append(np.stack([t_a, t_b], axis=1).reshape(-1, 3, 3))
    # long thin triangles: length U(2, 10), width length / 200
    j = np.arange(n_thin, dtype=np.uint32)
    c = np.stack([uniform(seed, 30, j) * 200.0 - 100.0, uniform(seed, 31, j) * 60.0,
                  uniform(seed, 32, j) * 200.0 - 100.0], axis=-1)
    u = unit_vectors(seed, 33, j)
    w = unit_vectors(seed, 35, j)
    w = w - (w * u).sum(axis=1, keepdims=True) * u
    w = w / np.sqrt(np.maximum((w * w).sum(axis=1, keepdims=True), 1e-30))
    length = 2.0 + 8.0 * uniform(seed, 37, j)
    half = (0.5 * length)[:, None] * u
    parts.append(np.stack([c - half, c + half, c + (length / 200.0)[:, None] * w], axis=1))
    tri = np.concatenate(parts, axis=0)
    n = tri.shape[0]
    vertices = _f32(tri.reshape(3 * n, 3))
    triangles = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return vertices, triangles


def rays_in_box(n: int, lo, hi, seed: int = 6, expand: float = 0.1):
    """Rays with origins uniform in the box [lo, hi] grown by `expand` of its
    extent on every side and directions uniform on the sphere: float32
    [n, 8] = origin xyz, 0, direction xyz, 0."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    ext = hi - lo
    lo2 = lo - expand * ext
    ext2 = ext * (1.0 + 2.0 * expand)
    i = np.arange(n, dtype=np.uint32)
    o = lo2 + ext2 * np.stack([uniform(seed, 40 + k, i) for k in range(3)], axis=-1)
    d = unit_vectors(seed, 43, i)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = _f32(o)
    r[:, 4:7] = _f32(d)
    return r


def quaternion_matrix(q):
    """3x3 rotation matrices of unit quaternions q [n, 4] (x, y, z, w)."""
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)


def instance_transforms(rot, scale, trans) -> np.ndarray:
    """Column-major f32 4x4 matrices x -> R (s x) + t, 16 floats per instance
    (glam's Mat4 layout: x_axis, y_axis, z_axis, w_axis columns)."""
    n = rot.shape[0]
    m = np.zeros((n, 4, 4), np.float64)  # [instance, column, row]
    for c in range(3):
        m[:, c, 0:3] = rot[:, :, c] * scale[:, None]
    m[:, 3, 0:3] = trans
    m[:, 3, 3] = 1.0
    return _f32(m.reshape(n, 16))


def instance_aabbs(mesh_bounds: np.ndarray, mesh_ids, transforms) -> np.ndarray:
    """World AABB of each instance as marigold's scene upload computes it
    (marigold/src/app/data/scene/model.rs:191-234), in f32: the 8 corners of
    the mesh's bounds as (x, y, z, 1) through the column-major matrix, each
    component ((c0 x + c1 y) + c2 z) + c3 * 1 with every product and sum
    rounded (glam 0.30 Mat4 * Vec4), then min/max over the corners in corner
    order with ties taking the later corner (SSE minps/maxps)."""
    b = np.asarray(mesh_bounds, np.float32)[np.asarray(mesh_ids)]
    m = np.asarray(transforms, np.float32).reshape(-1, 4, 4)  # [instance, column, row]
    lo = np.full((b.shape[0], 3), np.inf, np.float32)
    hi = np.full((b.shape[0], 3), -np.inf, np.float32)
    one = np.float32(1.0)
    for i in range(8):
        x = b[:, 3 if (i >> 2) & 1 else 0]
        y = b[:, 4 if (i >> 1) & 1 else 1]
        z = b[:, 5 if i & 1 else 2]
        w = ((m[:, 0, 0:3] * x[:, None] + m[:, 1, 0:3] * y[:, None]) + m[:, 2, 0:3] * z[:, None]) \
            + m[:, 3, 0:3] * one
        lo = np.where(lo < w, lo, w)
        hi = np.where(hi > w, hi, w)
    return np.concatenate([lo, hi], axis=1).astype(np.float32)


def batched_scene(seed: int = 3, n_meshes: int = 512, n_instances: int = 4096,
                  lo: int = 64, hi: int = 262144):
    """Many meshes plus instances: triangle counts log-uniform in [lo, hi];
    each mesh is random small triangles or a noisy icosphere (coin flip; the
    icosphere is subdivided to the first level with enough faces and trimmed);
    instances pick a mesh uniformly, a random rotation (normalised 4-D
    Gaussian quaternion), a uniform scale in [0.5, 2] and a translation uniform
    in [-100, 100]^3. Returns (meshes, bounds [M, 6], instance AABBs [I, 6])
    with meshes a list of (vertices float32 [V, 8], triangles uint32 [N, 3])."""
    m = np.arange(n_meshes, dtype=np.uint32)
    counts = np.rint(np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * uniform(seed, 1, m))).astype(np.int64)
    kind = uniform(seed, 2, m) < 0.5
    ico_cache = {}
    meshes = []
    for i in range(n_meshes):
        n = int(counts[i])
        if kind[i]:
            v, t = random_triangles(n, seed=10000 + i)
        else:
            level = 0
            while 20 * 4 ** level < n:
                level += 1
            if level not in ico_cache:
                ico_cache[level] = icosphere(level)
            p, f = ico_cache[level]
            r = 1.0 + 0.05 * value_noise(p, 20000 + i)
            v = pack_vertices(p * r[:, None])
            t = f[:n].astype(np.uint32)
        meshes.append((v, np.ascontiguousarray(t, dtype=np.uint32)))
    bounds = np.stack([mesh_bounds(v) for v, _ in meshes])
    ids, xf = scene_instances(seed, n_meshes, n_instances)
    inst = instance_aabbs(bounds, ids, xf)
    return meshes, bounds, inst


def scene_instances(seed: int, n_meshes: int, n_instances: int):
    """Instances of the batched scene: mesh ids (uint32 [I], uniform) and f32
    column-major transforms [I, 16] (rotation from a normalised 4-D Gaussian
    quaternion, uniform scale in [0.5, 2], translation uniform in
    [-100, 100]^3)."""
    j = np.arange(n_instances, dtype=np.uint32)
    ids = np.minimum((uniform(seed, 3, j) * n_meshes).astype(np.int64), n_meshes - 1).astype(np.uint32)
    q = np.stack([gaussian(seed, 10 + 2 * k, j) for k in range(4)], -1)
    q = q / np.sqrt((q * q).sum(axis=1, keepdims=True))
    scale = 0.5 + 1.5 * uniform(seed, 20, j)
    trans = np.stack([uniform(seed, 21 + k, j) * 200.0 - 100.0 for k in range(3)], -1)
    return ids, instance_transforms(quaternion_matrix(q), scale, trans)
