"""Seeded ray sets for traversal parity: shadow rays between voxel faces,
random segments, and degenerate rays along voxel faces, edges and corners
(the cases where the box test is rounding-sensitive)."""
import numpy as np

from cube_tracing import layouts as L


def _f32(a):
    return np.asarray(a, np.float32)


def ray_origin_offset(pos, n):
    """compute_ray_origin (primitives.glsl:233-257) in numpy float32."""
    pos = _f32(pos).copy()
    n = _f32(n)
    ioff = (n * np.float32(256.0)).astype(np.int32)
    bits = pos.view(np.int32)
    ipos = (bits + np.where(pos < 0, -ioff, ioff)).astype(np.int32).view(np.float32)
    fpos = (pos + n * np.float32(1.0 / 65536.0)).astype(np.float32)
    return np.where(np.abs(pos) < np.float32(1.0 / 32.0), fpos, ipos).astype(np.float32)


def _normalize(v):
    v = _f32(v)
    l = np.sqrt((v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2]).astype(np.float32))
    return (v / l[..., None]).astype(np.float32)


FACES = np.array([[-1, 0, 0], [1, 0, 0], [0, -1, 0], [0, 1, 0], [0, 0, -1], [0, 0, 1]], np.float32)


def face_points(scene, rng, idx):
    """A random point on a random face of voxels `idx`, pushed off the face
    twice as the shaders do, and the face normal."""
    e = np.float32(scene.voxel_extent)
    c = (scene.aabbs["minimum"][idx] + scene.aabbs["maximum"][idx]) * np.float32(0.5)
    f = FACES[rng.integers(0, 6, idx.shape[0])]
    uv = rng.uniform(-0.5, 0.5, (idx.shape[0], 3)).astype(np.float32) * e
    uv = uv * (1 - np.abs(f))
    p = (c + f * (e * np.float32(0.5)) + uv).astype(np.float32)
    return ray_origin_offset(ray_origin_offset(p, f), f), f


def shadow_rays(scene, n, seed):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, scene.voxel_count, n)
    P, _ = face_points(scene, rng, src)
    lights = rng.integers(0, scene.cube_lights.shape[0], n)
    lvox = scene.cube_lights["primitive_id"][lights].astype(np.int64)
    Q, _ = face_points(scene, rng, lvox)
    d = _normalize(Q - P)
    dist = np.sqrt(((P - Q) ** 2).sum(-1).astype(np.float32)).astype(np.float32)
    r = np.zeros(n, L.RAY_QUERY)
    r["origin"], r["direction"], r["distance"] = P, d, dist
    r["flags"] = L.QUERY_CHECK_TARGET * (rng.random(n) < 0.8)
    r["target_instance"] = 0
    r["target_primitive"] = lvox
    return r


def random_segments(scene, n, seed):
    rng = np.random.default_rng(seed)
    lo = scene.aabbs["minimum"].min(0) - 4
    hi = scene.aabbs["maximum"].max(0) + 4
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = _normalize(rng.normal(size=(n, 3)))
    r = np.zeros(n, L.RAY_QUERY)
    r["origin"], r["direction"] = o, d
    r["distance"] = rng.uniform(0.5, float(np.max(hi - lo)), n).astype(np.float32)
    return r


def degenerate_rays(scene, n, seed):
    """Axis-aligned rays on integer / half-integer planes, diagonals through
    edges and corners."""
    rng = np.random.default_rng(seed)
    lo = scene.aabbs["minimum"].min(0) - 2
    hi = scene.aabbs["maximum"].max(0) + 2
    dirs = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                     [1, 1, 0], [1, -1, 0], [0, 1, 1], [1, 0, -1], [1, 1, 1], [-1, 1, -1]], np.float32)
    d = _normalize(dirs[rng.integers(0, len(dirs), n)])
    o = np.floor(rng.uniform(lo, hi, (n, 3))).astype(np.float32)
    half = rng.random((n, 3)) < 0.3
    o = (o + half * np.float32(0.5)).astype(np.float32)
    r = np.zeros(n, L.RAY_QUERY)
    r["origin"], r["direction"] = o, d
    r["distance"] = np.float32(float(np.max(hi - lo)) * 2)
    return r


def camera_rays(scene, n, seed):
    rng = np.random.default_rng(seed)
    lo = scene.aabbs["minimum"].min(0)
    hi = scene.aabbs["maximum"].max(0)
    c = (lo + hi) * 0.5
    R = float(np.max(hi - lo))
    u = _normalize(rng.normal(size=(n, 3)))
    o = (c + u * R * rng.uniform(0.8, 1.5, (n, 1))).astype(np.float32)
    t = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    r = np.zeros(n, L.RAY_QUERY)
    r["origin"], r["direction"] = o, _normalize(t - o)
    r["distance"] = np.float32(1e9)
    return r
