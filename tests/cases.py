"""Workloads shared by the golden fixtures, the oracle tests and the GPU
parity tests: small seeded scenes the CPU oracle renders in seconds."""
import numpy as np

from cube_tracing import layouts as L
from cube_tracing import scenes


def build_case(name):
    """Returns (scene, width, height, camera list, renderer kwargs)."""
    if name == "grid16":
        sc = scenes.random_grid_scene(16, 0.3, emissive_fraction=0.05, seed=3)
        W, H = 36, 28  # not multiples of 8: exercises the TAA edge rule
        cams = scenes.camera_path("translate", 3, W, H, eye=(-4.0, 8.0, -4.0), target=(8.0, 8.0, 8.0),
                                  step=(0.1, 0.0, 0.0))
        return sc, W, H, cams, {}
    if name == "grid32_allfeatures":
        sc = scenes.random_grid_scene(32, 0.2, emissive_fraction=0.03, seed=11)
        pl = np.zeros(1, L.LIGHT)
        pl["position"] = (16.0, 40.0, 16.0)
        pl["emissive"] = (300.0, 300.0, 300.0)
        pl["instance_id"] = L.MAX_INSTANCES
        pl["primitive_id"] = L.MAX_PRIMITIVES
        pl["type"] = L.LIGHT_POINT
        el = np.zeros(1, L.LIGHT)
        el["emissive"] = (10.0, 10.0, 10.0)
        el["instance_id"] = L.MAX_INSTANCES
        el["primitive_id"] = L.MAX_PRIMITIVES
        el["type"] = L.LIGHT_ENV_MAP
        sc.point_lights, sc.env_lights = pl, el
        sc.light_config["point_light_count"] = 1
        sc.light_config["env_map_count"] = 1
        W, H = 40, 32
        cams = scenes.camera_path("translate", 3, W, H, eye=(-10.0, 20.0, -10.0), target=(16.0, 12.0, 16.0),
                                  step=(0.1, 0.0, 0.05))
        feats = L.RIS_POINT_LIGHT_BIT | L.RIS_ENV_LIGHT_BIT | L.RIS_CUBE_LIGHT_BIT
        return sc, W, H, cams, {"features": feats}
    if name == "terrain32":
        sc = scenes.heightfield_scene(32, base=8.0, amplitude=6.0, emissive_fraction=0.05, seed=5)
        W, H = 32, 32
        cams = scenes.camera_path("orbit", 3, W, H, center=(16.0, 8.0, 16.0), radius=40.0, elevation=25.0,
                                  deg_per_frame=1.0)
        return sc, W, H, cams, {}
    if name == "config0":
        # the small plain workload at full size: 64^3 grid, p = 0.3, 2% emissive
        # cubes U[1,10], albedo U[0.2,0.8]; camera at (-16,32,-16) looking at the
        # grid centre, 256x256, 60 deg, 8 frames moving 0.1 along +x; max depth
        # 4 with ReSTIR DI and PT.  The oracle runs the reference's compiled-in
        # reuse parameters (3-4 neighbours within 2-50 px, one spatial pass),
        # so the CUDA path runs the same.
        sc = scenes.random_grid_scene(64, 0.3, emissive_fraction=0.02, seed=0, albedo=(0.2, 0.8),
                                      radiance=(1.0, 10.0))
        pl = np.zeros(1, L.LIGHT)
        pl["position"] = (32.0, 96.0, 32.0)
        pl["emissive"] = (50.0, 50.0, 50.0)
        pl["instance_id"] = L.MAX_INSTANCES
        pl["primitive_id"] = L.MAX_PRIMITIVES
        pl["type"] = L.LIGHT_POINT
        sc.point_lights = pl
        sc.light_config["point_light_count"] = 1
        W, H = 256, 256
        cams = scenes.camera_path("translate", 8, W, H, eye=(-16.0, 32.0, -16.0), target=(32.0, 32.0, 32.0),
                                  step=(0.1, 0.0, 0.0))
        return sc, W, H, cams, {"indirect": True, "max_depth": 4}
    if name == "config0_spec":
        # the small plain workload exactly as specified: as "config0", but
        # without the point light, and with spatial reuse over 5 neighbours
        # in a 30-pixel radius (min = max for both, so the reference's
        # confidence and distance heuristics pick those values); one
        # temporal and one spatial pass, 32 cube-light candidates
        sc, W, H, cams, kw = build_case("config0")
        sc.point_lights = np.zeros(0, L.LIGHT)
        sc.light_config["point_light_count"] = 0
        kw = dict(kw, params={"min_num_of_neighbors": 5, "max_num_of_neighbors": 5, "min_neighbors_radius": 30.0,
                              "max_neighbors_radius": 30.0, "max_ris_cube_samples": 32, "spatial_passes": 1})
        return sc, W, H, cams, kw
    if name == "terrain32_rounds_pt":
        # the reuse parameters of the 1080p terrain workload at fixture size:
        # two DI spatial rounds (the intermediate -> current ping-pong), TAA
        # keeping 0.9 of the history, PT to depth 8
        sc, W, H, cams, kw = build_case("terrain32_pt")
        return sc, W, H, cams, dict(kw, max_depth=8, params={"spatial_passes": 2, "taa_alpha": 0.1})
    if name == "grid16_nbr5_pt":
        # five spatial neighbours in a fixed 30-pixel radius, three rounds
        # (an odd number of extra rounds ends in the current reservoirs)
        sc, W, H, cams, kw = build_case("grid16_pt")
        return sc, W, H, cams, dict(kw, params={"min_num_of_neighbors": 5, "max_num_of_neighbors": 5,
                                                "min_neighbors_radius": 30.0, "max_neighbors_radius": 30.0,
                                                "spatial_passes": 3})
    if name.endswith("_hybrid_pt"):
        # the hybrid shift (ct_params.pt_shift_mapping = CT_SHIFT_HYBRID) with
        # a 0.5-unit near-field distance: reconnection vertices at lengths 1-3,
        # the longer ones reached by replaying the prefix
        sc, W, H, cams, kw = build_case(name.replace("_hybrid_pt", "_pt"))
        params = dict(kw.get("params", {}), pt_shift_mapping=2, pt_near_field_distance=0.5)
        return sc, W, H, cams, dict(kw, params=params)
    if name == "grid16_materials_pt":
        # every material type of MATERIAL.type (shared.inl:295-298): the BRDFs
        # and pdfs of metal, dielectric and constant medium (mat.glsl:30-88,
        # light.glsl:200-229) next to Lambertian, under DI and PT
        sc, W, H, cams, kw = build_case("grid16_pt")
        rng = np.random.default_rng(23)
        m = sc.materials
        n = m.shape[0]
        m["type"] = np.arange(n, dtype=np.uint32) % 4
        m["roughness"] = rng.uniform(0.05, 1.0, n).astype(np.float32)
        m["specular"] = rng.uniform(0.0, 0.6, (n, 3)).astype(np.float32)
        m["ior"] = rng.uniform(1.1, 1.8, n).astype(np.float32)
        return sc, W, H, cams, kw
    if name in ("grid16_brdf", "grid16_materials_brdf_pt"):
        # BRDF-sampled RIS candidates (RIS_BRDF_BIT, restir_resampling.glsl:193-248)
        # with the reference app's one BRDF sample (BRDF_SAMPLING_COUNT,
        # shared.inl:31; main.cpp:1319)
        sc, W, H, cams, kw = build_case(name.replace("_brdf", ""))
        sc.light_config["brdf_count"] = 1
        kw = dict(kw, features=kw.get("features", L.RIS_CUBE_LIGHT_BIT) | L.RIS_BRDF_BIT)
        return sc, W, H, cams, kw
    if name == "glass_inside_brdf_pt":
        # the camera inside a dielectric voxel for two frames, then out
        # through its +x face into free space: in the first frames every
        # primary hit is one of the voxel's own faces seen from behind, and
        # the BRDF candidate's dielectric callable turns the first pass's hit
        # record (sample_material takes it inout, light.glsl:231), which the
        # RIS visibility pass and TEMPORAL_REUSE then use (rgen.glsl:255-262)
        sc, W, H, _, kw = build_case("grid16_materials_brdf_pt")
        lo = sc.aabbs["minimum"]
        occupied = {tuple(v) for v in np.floor(lo).astype(np.int64).tolist()}
        glass = (sc.materials["type"][sc.primitives["material_index"]] & 0xFF) == 2
        centre = np.float32(8.0)
        best = None
        for p in np.argsort(np.abs(lo - centre).sum(-1), kind="stable"):
            v = tuple(np.floor(lo[p]).astype(np.int64).tolist())
            if glass[p] and (v[0] + 1, v[1], v[2]) not in occupied and (v[0] + 2, v[1], v[2]) not in occupied:
                best = p
                break
        x1 = float(sc.aabbs["maximum"][best, 0])
        eye = (x1 - 0.15, float(lo[best, 1]) + 0.37, float(lo[best, 2]) + 0.61)
        target = (eye[0] + 10.0, eye[1] - 2.0, eye[2] + 3.0)
        cams = scenes.camera_path("translate", 3, W, H, eye=eye, target=target, step=(0.1, 0.0, 0.0))
        return sc, W, H, cams, kw
    if name == "instances16":
        # four instances over x slabs of one grid, each under its own TLAS
        # transform (INSTANCE.transform, accel_struct_mngr.cpp:1888-1889): a
        # whole-voxel translation, a fractional translation with a 0.3 rad
        # turn about y, the reference's 0.1 degree update turn (main.cpp:1377),
        # and a 0.4 rad turn about an oblique axis, whose off-diagonal terms
        # show the closest-hit shader's model-matrix indexing (rchit.glsl:29-33)
        sc = scenes.random_grid_scene(16, 0.25, emissive_fraction=0.06, seed=13)
        turns = [rotation((0.0, 1.0, 0.0), 0.0), rotation((0.0, 1.0, 0.0), 0.3),
                 rotation((0.0, 1.0, 0.0), np.radians(0.1)), rotation((1.0, 2.0, 2.0), 0.4)]
        moves = [(2.0, 0.0, -1.0), (1.25, -0.5, 3.75), (-2.0, 1.0, 0.0), (0.5, 0.25, -0.75)]
        sc = split_into_instances(sc, [4.0, 8.0, 12.0], turns, moves)
        W, H = 40, 30
        cams = scenes.camera_path("translate", 3, W, H, eye=(8.0, 26.0, 2.0), target=(8.0, 0.0, 9.0),
                                  step=(0.1, 0.0, 0.05))
        return sc, W, H, cams, {}
    if name == "room16_deep_pt":
        # a closed 16^3 room seen from inside: no path escapes, so paths run
        # to max depth 12 and the wavefront's last rounds (paths longer than
        # 8 bounces) are exercised
        sc = closed_room_scene(16, seed=9)
        W, H = 32, 24
        cams = scenes.camera_path("translate", 3, W, H, eye=(7.5, 8.5, 3.5), target=(8.0, 6.0, 14.0),
                                  step=(0.05, 0.0, 0.0))
        pl = np.zeros(1, L.LIGHT)
        pl["position"] = (8.0, 13.0, 8.0)
        pl["emissive"] = (30.0, 30.0, 30.0)
        pl["instance_id"] = L.MAX_INSTANCES
        pl["primitive_id"] = L.MAX_PRIMITIVES
        pl["type"] = L.LIGHT_POINT
        sc.point_lights = pl
        sc.light_config["point_light_count"] = 1
        return sc, W, H, cams, {"indirect": True, "max_depth": 12}
    if name == "vox_room":
        # a MagicaVoxel file made here (two models, RGBA palette, one emit
        # material), parsed and laid out as the reference's gvox loader does
        # with its maps' axis direction (map_loader.cpp:106-327)
        sc = scenes_from_vox_bytes(vox_room_bytes())
        W, H = 40, 30
        cams = scenes.camera_path("translate", 3, W, H, eye=(-6.0, 14.0, -6.0), target=(12.0, 4.0, 12.0),
                                  step=(0.1, 0.0, 0.05))
        return sc, W, H, cams, {}
    if name.endswith("_pt"):
        # the same workload with indirect illumination (ReSTIR PT); PT's next
        # event estimation samples point lights, so every PT case has one
        sc, W, H, cams, kw = build_case(name[:-3])
        if sc.light_config["point_light_count"] == 0:
            pl = np.zeros(1, L.LIGHT)
            pl["position"] = (8.0, 30.0, 8.0)
            pl["emissive"] = (200.0, 200.0, 200.0)
            pl["instance_id"] = L.MAX_INSTANCES
            pl["primitive_id"] = L.MAX_PRIMITIVES
            pl["type"] = L.LIGHT_POINT
            sc.point_lights = pl
            sc.light_config["point_light_count"] = 1
        kw = dict(kw, indirect=True, max_depth=4)
        return sc, W, H, cams, kw
    raise KeyError(name)


def vox_room_bytes(seed=7):
    """Two models over a 24 x 24 x 12 extent (MagicaVoxel z is up): a floor
    with two walls and a lit pillar in model 0, scattered boxes with emissive
    tops in model 1 on cells model 0 leaves empty."""
    from cube_tracing import vox
    rng = np.random.default_rng(seed)
    X, Y, Z = 24, 24, 12
    occ = np.zeros((X, Y, Z), np.uint8)
    occ[:, :, 0] = rng.integers(1, 5, (X, Y))                       # floor, colours 1-4
    occ[0, :, 1:9] = 5                                              # wall along y
    occ[:, 0, 1:7] = 6                                              # wall along x
    occ[12, 12, 1:8] = 7
    occ[12, 12, 8] = 9                                              # emissive cap
    m0 = np.argwhere(occ > 0)
    v0 = np.concatenate([m0, occ[occ > 0][:, None]], axis=1).astype(np.uint8)
    boxes = []
    for _ in range(10):
        x, y = rng.integers(3, 21, 2)
        h = int(rng.integers(1, 4))
        for z in range(1, h + 1):
            if occ[x, y, z] == 0:
                boxes.append((x, y, z, 8))
        if occ[x, y, h + 1] == 0:
            boxes.append((x, y, h + 1, 9 + int(rng.integers(0, 2))))
    v1 = np.unique(np.array(boxes, np.uint8), axis=0)
    pal = np.zeros((256, 4), np.uint8)
    pal[:, 3] = 255
    pal[:10, :3] = rng.integers(40, 230, (10, 3))
    pal[8, :3] = (255, 220, 160)  # colour index 9
    pal[9, :3] = (120, 200, 255)  # colour index 10
    return vox.write_vox([((X, Y, Z), v0), ((X, Y, Z), v1)], pal, emissive=(9, 10))


def closed_room_scene(edge=16, seed=0, interior=0.08, emissive_fraction=0.04):
    """The six walls of an edge^3 box plus scattered interior voxels (none
    within 2 cells of the room's front third centre line, where the camera
    stands); 4% of the voxels emit."""
    rng = np.random.default_rng(seed)
    g = np.arange(edge)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    wall = (x == 0) | (y == 0) | (z == 0) | (x == edge - 1) | (y == edge - 1) | (z == edge - 1)
    clear = (np.abs(x - 7.5) < 3) & (np.abs(y - 8.5) < 3) & (z < 7)
    occ = wall | ((rng.random(wall.shape) < interior) & ~clear)
    coords = np.argwhere(occ)[:, ::-1].astype(np.int32)
    n = coords.shape[0]
    emissive = rng.random(n) < emissive_fraction
    pal = rng.uniform(0.3, 0.8, size=(16, 3)).astype(np.float32)
    idx = rng.integers(0, 16, size=n).astype(np.uint32)
    rad = rng.uniform(1.0, 5.0, size=(int(emissive.sum()), 3)).astype(np.float32)
    return scenes._build(coords, emissive, pal, idx, rad, 1.0, (edge, edge, edge), f"room{edge}", {"seed": seed})


def rotation(axis, angle):
    """3x3 float32 rotation by `angle` radians about `axis` (Rodrigues)."""
    k = np.asarray(axis, np.float64)
    k = k / np.linalg.norm(k)
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    return (np.eye(3) + np.sin(angle) * K + (1.0 - np.cos(angle)) * K @ K).astype(np.float32)


def split_into_instances(sc, cuts, turns, moves):
    """The one-instance scene `sc` as len(cuts) + 1 instances: voxels with
    minimum x below cuts[0], then below cuts[1], ..., each group on its own
    contiguous primitive range in the same object space, with the transform
    turns[i] (a 3x3 rotation) then translate(moves[i]).  Cube lights follow
    their voxels; their positions are the voxels' world-space centres."""
    xs = sc.aabbs["minimum"][:, 0]
    group = np.searchsorted(np.asarray(cuts, np.float32), xs, side="right")
    order = np.argsort(group, kind="stable")
    new_of_old = np.empty_like(order)
    new_of_old[order] = np.arange(order.size)
    aabbs = sc.aabbs[order].copy()
    prims = sc.primitives[order].copy()
    g = group[order]
    inst = np.zeros(len(cuts) + 1, L.INSTANCE)
    mats = []
    for i in range(inst.shape[0]):
        idx = np.nonzero(g == i)[0]
        inst["first_primitive_index"][i] = idx[0] if idx.size else 0
        inst["primitive_count"][i] = idx.size
        m = np.eye(4, dtype=np.float32)
        m[:3, :3] = turns[i]
        m[:3, 3] = np.asarray(moves[i], np.float32)
        inst["transform"][i] = m.reshape(-1, order="F")
        mats.append(m)
    lights = sc.cube_lights.copy()
    for li in range(lights.shape[0]):
        new = int(new_of_old[int(lights["primitive_id"][li])])
        i = int(g[new])
        lights["instance_id"][li] = i
        lights["primitive_id"][li] = new - int(inst["first_primitive_index"][i])
        centre = (aabbs["minimum"][new] + aabbs["maximum"][new]) * np.float32(0.5)
        lights["position"][li] = (mats[i] @ np.append(centre, np.float32(1.0)))[:3]
    sc.instances, sc.aabbs, sc.primitives, sc.cube_lights = inst, aabbs, prims, lights
    return sc


def scenes_from_vox_bytes(data):
    from cube_tracing import vox
    models, pal, em = vox.read_vox(data)
    return vox.scene_from_vox(models, pal, em, 1.0, "X_BOTTOM_TOP", "vox_room")


CASES = ["grid16", "grid32_allfeatures", "terrain32", "grid16_brdf", "instances16"]
PT_CASES = ["grid16_pt", "grid32_allfeatures_pt", "terrain32_pt", "grid16_materials_pt", "vox_room_pt",
            "grid16_materials_brdf_pt", "room16_deep_pt", "glass_inside_brdf_pt",
            "instances16_pt", "terrain32_rounds_pt", "grid16_nbr5_pt", "grid16_hybrid_pt", "instances16_hybrid_pt",
            "grid16_materials_hybrid_pt", "room16_deep_hybrid_pt", "terrain32_hybrid_pt"]

FRAME_KEYS = ["di", "intermediate_reservoir", "previous_reservoir", "velocity"]
PT_KEYS = ["output_path_reservoir", "temporal_path_reservoir", "indirect_color"]


def frame_keys(name):
    return FRAME_KEYS + (PT_KEYS if name.endswith("_pt") else [])
