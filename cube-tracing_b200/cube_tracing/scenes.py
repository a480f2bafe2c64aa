"""Seeded synthetic voxel scenes and cameras for the hot-path workloads.

Scenes are built the way the reference's MagicaVoxel loader lays them out
(src/gvox/map_loader.cpp:205-296): one AABB per voxel (minimum = integer *
VOXEL_EXTENT, maximum = minimum + VOXEL_EXTENT), Lambertian materials
(type 0, roughness 1, ior 1, dissolve 1, illum 3), and one cube light per
emissive voxel whose LIGHT.position is the voxel centre, LIGHT.size the voxel
edge and LIGHT.instance_info the voxel's (instance, primitive) id; the
voxel's PRIMITIVE.light_index points at that light, other voxels carry
0xFFFFFFFF.

  random_grid_scene  -- an edge^3 grid with every cell occupied i.i.d.
                        (the 64^3, p=0.3 workload and the many-view sets)
  heightfield_scene  -- terrain filled below h(x,z) = base + amp * noise,
                        noise = 4-octave seeded value noise in [-1, 1]
                        (the 256^3 terrain workload)

Cameras follow the reference's conventions (src/camera.h:75-97 via glm):
right-handed look-at view, perspective with a [0,1] depth range, and the
Vulkan y flip applied to the inverse projection (src/main.cpp:1460).
"""
from dataclasses import dataclass, field
import math

import numpy as np

from . import layouts as L


@dataclass
class Scene:
    instances: np.ndarray
    aabbs: np.ndarray
    primitives: np.ndarray
    materials: np.ndarray
    cube_lights: np.ndarray
    point_lights: np.ndarray
    env_lights: np.ndarray
    light_config: np.ndarray
    voxel_extent: float
    grid_edge: tuple
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def voxel_count(self):
        return int(self.aabbs.shape[0])


def _identity():
    return np.eye(4, dtype=np.float32).reshape(-1, order="F")


def _build(coords, emissive_mask, albedo_pal, albedo_idx, radiance, voxel_extent, grid_edge, name, meta):
    n = coords.shape[0]
    e = np.float32(voxel_extent)
    aabbs = np.zeros(n, L.AABB)
    c = coords.astype(np.float32)
    aabbs["minimum"] = c * e
    aabbs["maximum"] = (c + np.float32(1.0)) * e

    n_pal = albedo_pal.shape[0]
    light_vox = np.nonzero(emissive_mask)[0]
    n_lights = light_vox.shape[0]
    materials = np.zeros(n_pal + n_lights, L.MATERIAL)
    materials["type"] = 0
    materials["shininess"] = 1.0
    materials["roughness"] = 1.0
    materials["ior"] = 1.0
    materials["dissolve"] = 1.0
    materials["illum"] = 3
    materials["diffuse"][:n_pal] = albedo_pal
    materials["diffuse"][n_pal:] = albedo_pal[albedo_idx[light_vox]]
    materials["emission"][n_pal:] = radiance

    primitives = np.zeros(n, L.PRIMITIVE)
    primitives["material_index"] = albedo_idx.astype(np.uint32)
    primitives["light_index"] = np.uint32(0xFFFFFFFF)
    primitives["material_index"][light_vox] = n_pal + np.arange(n_lights, dtype=np.uint32)
    primitives["light_index"][light_vox] = np.arange(n_lights, dtype=np.uint32)

    lights = np.zeros(n_lights, L.LIGHT)
    lights["position"] = c[light_vox] * e + e * np.float32(0.5)
    lights["emissive"] = radiance
    lights["instance_id"] = 0
    lights["primitive_id"] = light_vox.astype(np.uint32)
    lights["size"] = e
    lights["type"] = L.LIGHT_CUBE

    inst = np.zeros(1, L.INSTANCE)
    inst["transform"][0] = _identity()
    inst["first_primitive_index"] = 0
    inst["primitive_count"] = n

    cfg = np.zeros(1, L.LIGHT_CONFIG)
    cfg["cube_light_count"] = n_lights
    cfg["cube_light_pdf"] = 1.0 / max(n_lights, 1)
    cfg["light_count"] = n_lights

    return Scene(inst, aabbs, primitives, materials, lights, np.zeros(0, L.LIGHT), np.zeros(0, L.LIGHT), cfg,
                 float(voxel_extent), grid_edge, name, meta)


def random_grid_scene(edge=64, occupancy=0.3, emissive_fraction=0.02, seed=0, albedo=(0.2, 0.8),
                      radiance=(1.0, 10.0), palette=256, voxel_extent=1.0):
    """edge^3 grid, each cell occupied with probability `occupancy`;
    `emissive_fraction` of the occupied cells are cube lights with RGB radiance
    U[radiance], the rest Lambertian with per-channel albedo U[albedo] drawn
    from a palette of `palette` materials.  Voxels are ordered x fastest,
    then y, then z."""
    rng = np.random.default_rng(seed)
    occ = rng.random((edge, edge, edge), dtype=np.float32) < occupancy  # [z, y, x]
    zyx = np.argwhere(occ)
    coords = zyx[:, ::-1].astype(np.int32)
    n = coords.shape[0]
    emissive = rng.random(n) < emissive_fraction
    pal = rng.uniform(albedo[0], albedo[1], size=(palette, 3)).astype(np.float32)
    idx = rng.integers(0, palette, size=n).astype(np.uint32)
    rad = rng.uniform(radiance[0], radiance[1], size=(int(emissive.sum()), 3)).astype(np.float32)
    return _build(coords, emissive, pal, idx, rad, voxel_extent, (edge, edge, edge), f"grid{edge}_p{occupancy}",
                  {"seed": seed, "occupancy": occupancy})


def value_noise_2d(shape, seed, octaves=4, base_period=64.0):
    """Seeded value noise in [-1, 1]: random lattice values, smoothstep
    bilinear interpolation, `octaves` octaves with doubling frequency and
    halving amplitude, normalised by the amplitude sum."""
    rng = np.random.default_rng(seed)
    nz, nx = shape
    zz, xx = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    total = np.zeros(shape, np.float64)
    amp_sum = 0.0
    amp = 1.0
    period = base_period
    for _ in range(octaves):
        gz = int(math.ceil(nz / period)) + 2
        gx = int(math.ceil(nx / period)) + 2
        lattice = rng.uniform(-1.0, 1.0, size=(gz, gx))
        fz, fx = zz / period, xx / period
        iz, ix = np.floor(fz).astype(np.int64), np.floor(fx).astype(np.int64)
        tz, tx = fz - iz, fx - ix
        sz, sx = tz * tz * (3 - 2 * tz), tx * tx * (3 - 2 * tx)
        v00 = lattice[iz, ix]
        v01 = lattice[iz, ix + 1]
        v10 = lattice[iz + 1, ix]
        v11 = lattice[iz + 1, ix + 1]
        v0 = v00 + (v01 - v00) * sx
        v1 = v10 + (v11 - v10) * sx
        total += amp * (v0 + (v1 - v0) * sz)
        amp_sum += amp
        amp *= 0.5
        period *= 0.5
    return total / amp_sum


def heightfield_scene(edge=256, base=64.0, amplitude=48.0, emissive_fraction=0.005, seed=1, albedo=(0.1, 0.9),
                      radiance=(2.0, 20.0), palette=256, voxel_extent=1.0):
    """edge x edge columns filled below h(x,z) = base + amplitude * noise(x,z)
    (height clipped to [1, edge]).  `emissive_fraction` of the surface voxels
    (voxels with at least one empty face neighbour) are cube lights."""
    rng = np.random.default_rng(seed)
    h = base + amplitude * value_noise_2d((edge, edge), seed)
    h = np.clip(np.floor(h), 1, edge).astype(np.int32)  # [z, x] column heights
    # voxels (x, y, z) with y < h[z, x]; order: x fastest, then y, then z
    counts = h.reshape(-1)
    zz, xx = np.meshgrid(np.arange(edge, dtype=np.int32), np.arange(edge, dtype=np.int32), indexing="ij")
    col_z = np.repeat(zz.reshape(-1), counts)
    col_x = np.repeat(xx.reshape(-1), counts)
    starts = np.cumsum(counts) - counts
    y = np.arange(counts.sum(), dtype=np.int64) - np.repeat(starts, counts)
    order = np.lexsort((col_x, y, col_z))
    coords = np.stack([col_x[order], y[order].astype(np.int32), col_z[order]], axis=1)
    # surface: top voxel of a column, or a side face above the neighbour column
    hp = np.pad(h, 1, constant_values=0)
    hz = coords[:, 2] + 1
    hx = coords[:, 0] + 1
    yy = coords[:, 1]
    min_nb = np.minimum.reduce([hp[hz - 1, hx], hp[hz + 1, hx], hp[hz, hx - 1], hp[hz, hx + 1]])
    surface = (yy == h[coords[:, 2], coords[:, 0]] - 1) | (yy >= min_nb)
    n = coords.shape[0]
    emissive = np.zeros(n, bool)
    surf_idx = np.nonzero(surface)[0]
    emissive[surf_idx[rng.random(surf_idx.shape[0]) < emissive_fraction]] = True
    pal = rng.uniform(albedo[0], albedo[1], size=(palette, 3)).astype(np.float32)
    idx = rng.integers(0, palette, size=n).astype(np.uint32)
    rad = rng.uniform(radiance[0], radiance[1], size=(int(emissive.sum()), 3)).astype(np.float32)
    return _build(coords, emissive, pal, idx, rad, voxel_extent, (edge, edge, edge), f"terrain{edge}",
                  {"seed": seed, "surface_voxels": int(surface.sum())})


# ---------------------------------------------------------------------------
# cameras

def look_at_rh(eye, center, up=(0.0, 1.0, 0.0)):
    eye, center, up = (np.asarray(v, np.float64) for v in (eye, center, up))
    f = center - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, u, -f
    m[0, 3], m[1, 3], m[2, 3] = -s @ eye, -u @ eye, f @ eye
    return m  # row-major math matrix


def perspective_rh_zo(fovy, aspect, near, far):
    t = math.tan(fovy / 2.0)
    m = np.zeros((4, 4))
    m[0, 0] = 1.0 / (aspect * t)
    m[1, 1] = 1.0 / t
    m[2, 2] = far / (near - far)
    m[3, 2] = -1.0
    m[2, 3] = -(far * near) / (far - near)
    return m


def col_major(m):
    return np.asarray(m, np.float64).astype(np.float32).reshape(-1, order="F")


def camera_matrices(eye, center, width, height, fovy_deg=60.0, near=0.1, far=10000.0):
    """(inv_view, inv_proj) as column-major float32[16], inv_proj with the
    Vulkan y flip (element [1][1] negated)."""
    view = look_at_rh(eye, center)
    proj = perspective_rh_zo(math.radians(fovy_deg), width / height, near, far)
    inv_view = np.linalg.inv(view)
    inv_proj = np.linalg.inv(proj)
    inv_proj[1, 1] *= -1.0
    return col_major(inv_view), col_major(inv_proj)


def camera_path(kind, n_frames, width, height, **kw):
    """List of (inv_view, inv_proj) per frame.
    kind 'translate': eye moves +step along x each frame (the 64^3 workload:
    eye (-16,32,-16) looking at (32,32,32), 0.1 units per frame).
    kind 'orbit': eye circles the centre at a fixed height."""
    out = []
    if kind == "translate":
        eye = np.array(kw.get("eye", (-16.0, 32.0, -16.0)))
        target = np.array(kw.get("target", (32.0, 32.0, 32.0)))
        step = np.array(kw.get("step", (0.1, 0.0, 0.0)))
        for f in range(n_frames):
            out.append(camera_matrices(eye + f * step, target + f * step, width, height, kw.get("fovy", 60.0)))
    elif kind == "orbit":
        c = np.array(kw.get("center", (128.0, 48.0, 128.0)))
        r = kw.get("radius", 240.0)
        h = kw.get("elevation", 150.0)
        dphi = math.radians(kw.get("deg_per_frame", 0.5))
        phi0 = math.radians(kw.get("phi0", 225.0))
        for f in range(n_frames):
            phi = phi0 + f * dphi
            eye = c + np.array([r * math.cos(phi), h, r * math.sin(phi)])
            out.append(camera_matrices(eye, c, width, height, kw.get("fovy", 60.0)))
    else:
        raise ValueError(kind)
    return out
