"""Seeded random frame cases for the parity sweep: random grids,
heightfields and multi-model .vox scenes, optionally split into several
instances under random TLAS transforms (translations, turns about random
axes), random light types, BRDF candidates and material types, DI alone or
with PT, TAA on or off, the sky's time of day, and an erase between frames
2 and 3.  Case k draws everything from numpy's default_rng(5000 + k)."""
import numpy as np

from cube_tracing import layouts as L
from cube_tracing import scenes


def split_instances(sc, k, rng, rotate=False, integer=True):
    """The one-instance scene `sc` as up to k instances: contiguous x slabs
    of its voxels cut at random voxel planes, each with a random translation
    (whole voxels, or with a fractional part) and, with `rotate`, a turn by
    up to 0.7 rad about a random axis.  Cube lights follow their voxels;
    their positions are the voxels' world-space centres."""
    lo = sc.aabbs["minimum"]
    xs = lo[:, 0]
    cuts = np.sort(rng.choice(np.unique(xs), size=min(k - 1, max(len(np.unique(xs)) - 1, 0)), replace=False))
    group = np.searchsorted(cuts, xs, side="right")
    order = np.argsort(group, kind="stable")
    new_of_old = np.empty_like(order)
    new_of_old[order] = np.arange(order.size)
    aabbs = sc.aabbs[order].copy()
    prims = sc.primitives[order].copy()
    g = group[order]
    n_inst = int(g.max()) + 1
    inst = np.zeros(n_inst, L.INSTANCE)
    mats = []
    for i in range(n_inst):
        idx = np.nonzero(g == i)[0]
        inst["first_primitive_index"][i] = idx[0] if idx.size else 0
        inst["primitive_count"][i] = idx.size
        m = np.eye(4, dtype=np.float32)
        if rotate and rng.random() < 0.7:
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            a = float(rng.uniform(-0.7, 0.7))
            K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            m[:3, :3] = (np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K).astype(np.float32)
        t = rng.integers(-3, 4, 3).astype(np.float32)
        if not integer:
            t = t + rng.uniform(-0.5, 0.5, 3).astype(np.float32)
        m[:3, 3] = t
        inst["transform"][i] = m.reshape(-1, order="F")
        mats.append(m)
    lights = sc.cube_lights.copy()
    for li in range(lights.shape[0]):
        new = int(new_of_old[int(lights["primitive_id"][li])])
        i = int(g[new])
        lights["instance_id"][li] = i
        lights["primitive_id"][li] = new - int(inst["first_primitive_index"][i])
        centre = (aabbs["minimum"][new] + aabbs["maximum"][new]) * np.float32(0.5)
        lights["position"][li] = (mats[i] @ np.append(centre, np.float32(1.0)).astype(np.float32))[:3]
    sc.instances, sc.aabbs, sc.primitives, sc.cube_lights = inst, aabbs, prims, lights
    return sc


def make_case(k, big=False, instances=True, rotate=True, sky=True):
    """Case k: (scene, W, H, cameras, renderer kwargs, edit) where edit is
    None or (pixel, half window) of an erase before frame 2."""
    rng = np.random.default_rng(5000 + k)
    edge = int(rng.integers(24, 65)) if big else int(rng.integers(8, 25))
    if rng.random() < 0.2:
        from cube_tracing import vox
        models = []
        for _ in range(int(rng.integers(1, 4))):
            sz = tuple(int(v) for v in rng.integers(4, edge + 1, 3))
            cnt = int(rng.integers(10, sz[0] * sz[1] * sz[2] // 3 + 11))
            xyz = np.stack([rng.integers(0, sz[a], cnt) for a in range(3)], 1)
            col = rng.integers(1, 12, (cnt, 1))
            models.append((sz, np.concatenate([xyz, col], 1).astype(np.uint8)))
        pal = np.zeros((256, 4), np.uint8)
        pal[:, 3] = 255
        pal[:16, :3] = rng.integers(30, 255, (16, 3))
        sc = vox.scene_from_vox(*vox.read_vox(vox.write_vox(models, pal, emissive=(9, 10, 11))), 1.0,
                                ["X_BOTTOM_TOP", "Z_BOTTOM_TOP", "Y_TOP_BOTTOM"][int(rng.integers(0, 3))])
    elif rng.random() < 0.3:
        sc = scenes.heightfield_scene(edge, base=edge / 3, amplitude=edge / 4, emissive_fraction=0.05, seed=k)
    else:
        sc = scenes.random_grid_scene(edge, float(rng.uniform(0.1, 0.5)),
                                      emissive_fraction=float(rng.uniform(0.02, 0.1)), seed=k)
    if instances and sc.instances.shape[0] == 1:
        sc = split_instances(sc, int(rng.integers(2, 5)), rng, rotate=rotate, integer=rng.random() < 0.5)
    feats = L.RIS_CUBE_LIGHT_BIT
    indirect = bool(rng.random() < 0.6)
    if rng.random() < 0.5 or indirect:
        pl = np.zeros(1, L.LIGHT)
        pl["position"] = rng.uniform(0, edge, 3) + np.array([0, edge, 0])
        pl["emissive"] = rng.uniform(50, 300)
        pl["instance_id"] = L.MAX_INSTANCES
        pl["primitive_id"] = L.MAX_PRIMITIVES
        pl["type"] = L.LIGHT_POINT
        sc.point_lights = pl
        sc.light_config["point_light_count"] = 1
        if rng.random() < 0.5:
            feats |= L.RIS_POINT_LIGHT_BIT
    if rng.random() < 0.3:
        el = np.zeros(1, L.LIGHT)
        el["emissive"] = rng.uniform(1, 10)
        el["instance_id"] = L.MAX_INSTANCES
        el["primitive_id"] = L.MAX_PRIMITIVES
        el["type"] = L.LIGHT_ENV_MAP
        sc.env_lights = el
        sc.light_config["env_map_count"] = 1
        feats |= L.RIS_ENV_LIGHT_BIT
    if rng.random() < 0.3:
        sc.light_config["brdf_count"] = 1
        feats |= L.RIS_BRDF_BIT
    if rng.random() < 0.3:
        m = sc.materials
        m["type"] = rng.integers(0, 4, m.shape[0]).astype(np.uint32)
        m["roughness"] = rng.uniform(0.05, 1, m.shape[0])
        m["ior"] = rng.uniform(1.1, 1.8, m.shape[0])
        m["specular"] = rng.uniform(0, 0.6, (m.shape[0], 3))
    W, H = ((int(rng.integers(48, 129)), int(rng.integers(40, 100))) if big
            else (int(rng.integers(12, 48)), int(rng.integers(12, 40))))
    edit = rng.random() < 0.4
    pix = (int(rng.integers(0, W)), int(rng.integers(0, H)))
    win = int(rng.integers(0, 6))
    c = np.array([edge / 2] * 3)
    eye = c + rng.normal(size=3) * edge * 1.2 + np.array([0, edge * 0.5, 0])
    cams = scenes.camera_path("translate", 5 if edit else 3, W, H, eye=tuple(eye), target=tuple(c),
                              step=tuple(rng.normal(size=3) * 0.1))
    kw = {"features": feats}
    if sky:
        kw.update(taa=bool(rng.random() < 0.7), sky_time=float(rng.uniform(0.0, 1.0)),
                  is_afternoon=int(rng.integers(0, 2)))
    if indirect:
        kw.update(indirect=True, max_depth=int(rng.integers(2, 7)))
    return sc, W, H, cams, kw, ((pix, win) if edit else None)
