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


def instance_of(scene, idx):
    """(instance, primitive id within it) of global primitive indices."""
    first = scene.instances["first_primitive_index"].astype(np.int64)
    count = scene.instances["primitive_count"].astype(np.int64)
    inst = np.zeros(idx.shape[0], np.int64)
    for i in range(first.shape[0]):
        inst[(idx >= first[i]) & (idx < first[i] + count[i])] = i
    return inst, (idx - first[inst]).astype(np.uint32)


def _to_world(scene, inst, v, w):
    """Object-space vectors `v` (w = 1 points, 0 directions) of instances
    `inst` in world space; identity instances pass them through untouched."""
    out = _f32(v).copy()
    for i in np.unique(inst):
        m = scene.instances["transform"][i].reshape(4, 4, order="F").astype(np.float32)
        if np.array_equal(m, np.eye(4, dtype=np.float32)):
            continue
        sel = inst == i
        h = np.concatenate([out[sel], np.full((int(sel.sum()), 1), np.float32(w))], axis=1).astype(np.float32)
        out[sel] = (h @ m.T)[:, :3]
    return out.astype(np.float32)


def world_bounds(scene):
    """Corners of the scene's world-space bounding box."""
    lo, hi = scene.aabbs["minimum"], scene.aabbs["maximum"]
    inst, _ = instance_of(scene, np.arange(lo.shape[0]))
    pts = [_to_world(scene, inst, np.stack([(lo, hi)[a][:, 0], (lo, hi)[b][:, 1], (lo, hi)[c][:, 2]], 1), 1.0)
           for a in (0, 1) for b in (0, 1) for c in (0, 1)]
    pts = np.concatenate(pts)
    return pts.min(0), pts.max(0)


def face_points(scene, rng, idx):
    """A random point on a random face of voxels `idx`, pushed off the face
    twice as the shaders do, and the face normal (world space)."""
    e = np.float32(scene.voxel_extent)
    c = (scene.aabbs["minimum"][idx] + scene.aabbs["maximum"][idx]) * np.float32(0.5)
    f = FACES[rng.integers(0, 6, idx.shape[0])]
    uv = rng.uniform(-0.5, 0.5, (idx.shape[0], 3)).astype(np.float32) * e
    uv = uv * (1 - np.abs(f))
    p = (c + f * (e * np.float32(0.5)) + uv).astype(np.float32)
    inst, _ = instance_of(scene, idx)
    p, f = _to_world(scene, inst, p, 1.0), _to_world(scene, inst, f, 0.0)
    return ray_origin_offset(ray_origin_offset(p, f), f), f


def shadow_rays(scene, n, seed):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, scene.voxel_count, n)
    P, _ = face_points(scene, rng, src)
    lights = rng.integers(0, scene.cube_lights.shape[0], n)
    cl = scene.cube_lights[lights]
    lvox = scene.instances["first_primitive_index"][cl["instance_id"]].astype(np.int64) + cl["primitive_id"]
    Q, _ = face_points(scene, rng, lvox)
    d = _normalize(Q - P)
    dist = np.sqrt(((P - Q) ** 2).sum(-1).astype(np.float32)).astype(np.float32)
    r = np.zeros(n, L.RAY_QUERY)
    r["origin"], r["direction"], r["distance"] = P, d, dist
    r["flags"] = L.QUERY_CHECK_TARGET * (rng.random(n) < 0.8)
    r["target_instance"], r["target_primitive"] = instance_of(scene, lvox)
    return r


def random_segments(scene, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = world_bounds(scene)
    lo, hi = lo - 4, hi + 4
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
    lo, hi = world_bounds(scene)
    lo, hi = lo - 2, hi + 2
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
    lo, hi = world_bounds(scene)
    c = (lo + hi) * 0.5
    R = float(np.max(hi - lo))
    u = _normalize(rng.normal(size=(n, 3)))
    o = (c + u * R * rng.uniform(0.8, 1.5, (n, 1))).astype(np.float32)
    t = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    r = np.zeros(n, L.RAY_QUERY)
    r["origin"], r["direction"] = o, _normalize(t - o)
    r["distance"] = np.float32(1e9)
    return r
