"""numpy dtypes for the reference GPU structs (src/shaders/shared.inl).

These mirror include/ct.h field for field; `tests/test_layouts.py` checks the
sizes against both the C header (via the library's own static_asserts) and
the oracle's compiled view of shared.inl.
"""
import numpy as np

f3 = ("<f4", (3,))

AABB = np.dtype([("minimum", *f3), ("maximum", *f3)])
INSTANCE = np.dtype([("transform", "<f4", (16,)), ("first_primitive_index", "<u4"), ("primitive_count", "<u4")])
PRIMITIVE = np.dtype([("material_index", "<u4"), ("light_index", "<u4")])
MATERIAL = np.dtype([
    ("type", "<u4"), ("ambient", *f3), ("diffuse", *f3), ("specular", *f3), ("transmittance", *f3),
    ("emission", *f3), ("shininess", "<f4"), ("roughness", "<f4"), ("ior", "<f4"), ("dissolve", "<f4"),
    ("illum", "<i4"),
])
LIGHT = np.dtype([
    ("position", *f3), ("emissive", *f3), ("instance_id", "<u4"), ("primitive_id", "<u4"),
    ("size", "<f4"), ("type", "<u4"),
])
LIGHT_CONFIG = np.dtype([
    ("point_light_count", "<u4"), ("point_light_pdf", "<f4"), ("cube_light_count", "<u4"), ("cube_light_pdf", "<f4"),
    ("sphere_light_count", "<u4"), ("sphere_light_pdf", "<f4"), ("analytic_light_count", "<u4"),
    ("analytic_light_pdf", "<f4"), ("env_map_count", "<u4"), ("env_map_pdf", "<f4"), ("brdf_count", "<u4"),
    ("brdf_pdf", "<f4"), ("light_count", "<u4"),
])
RESERVOIR = np.dtype([
    ("Y", "<u4"), ("l_type", "<u4"), ("seed", "<u4"), ("W_y", "<f4"), ("W_sum", "<f4"), ("M", "<f4"), ("F", *f3),
])
DI_INFO = np.dtype([
    ("position", *f3), ("distance", "<f4"), ("normal", *f3), ("ray_origin", *f3), ("seed", "<u4"),
    ("instance_id", "<u4"), ("primitive_id", "<u4"), ("mat_index", "<u4"), ("confidence", "<f4"),
])
VELOCITY = np.dtype([("velocity", "<f4", (2,))])
PATH_RESERVOIR = np.dtype([
    ("M", "<f4"), ("weight", "<f4"), ("path_flags", "<u4"), ("rc_random_seed", "<u4"), ("F", *f3),
    ("light_pdf", "<f4"), ("cached_jacobian", *f3), ("init_random_seed", "<u4"), ("rc_instance_id", "<u4"),
    ("rc_primitive_id", "<u4"), ("rc_hit", *f3), ("rc_vertex_wi", *f3), ("rc_vertex_irradiance", *f3),
])
CAMERA_VIEW = np.dtype([
    ("inv_view", "<f4", (16,)), ("inv_proj", "<f4", (16,)), ("defocus_angle", "<f4"), ("focus_dist", "<f4"),
    ("prev_inv_view", "<f4", (16,)), ("prev_inv_proj", "<f4", (16,)),
])
STATUS = np.dtype({
    "names": ["resolution", "frame_number", "num_accumulated_frames", "pixel", "is_active", "light_config_address",
              "obj_count", "time", "is_afternoon", "max_depth", "brush_config_address", "brush_counter_address",
              "instance_bitmask_address", "primitive_bitmask_address"],
    "formats": [("<u4", (2,)), "<u4", "<u8", ("<u4", (2,)), "<u4", "<u8", "<u4", "<f4", "<u4", "<u4", "<u8", "<u8",
                "<u8", "<u8"],
    "offsets": [0, 8, 16, 24, 32, 40, 48, 52, 56, 60, 64, 72, 80, 88],
    "itemsize": 96,
})
WORLD_FIELDS = ["instance_address", "instance_address_prev", "primitive_address", "primitive_address_prev",
                "aabb_address", "aabb_address_prev", "remapped_primitive_address", "remapped_cube_light_address",
                "material_address", "point_light_address", "cube_light_address", "env_light_address"]
WORLD = np.dtype([(n, "<u8") for n in WORLD_FIELDS])
RESTIR_FIELDS = ["previous_reservoir_address", "intermediate_reservoir_address", "reservoir_address",
                 "previous_di_address", "di_address", "velocity_address", "output_path_reservoir_address",
                 "temporal_path_reservoir_address", "indirect_color_address"]
RESTIR = np.dtype([(n, "<u8") for n in RESTIR_FIELDS])
BRUSH_CONFIG = np.dtype([("brush_type", "<u4"), ("brush_size", "<f4", (3,)), ("brush_pixel_size", "<u4", (3,))])
BRUSH_COUNTER = np.dtype([("instance_count", "<u4"), ("primitive_count", "<u4")])

RAY_QUERY = np.dtype([("origin", *f3), ("distance", "<f4"), ("direction", *f3), ("flags", "<u4"),
                      ("target_instance", "<u4"), ("target_primitive", "<u4")])
RAY_HIT = np.dtype([("instance_id", "<u4"), ("primitive_id", "<u4"), ("t", "<f4"), ("_pad", "<u4")])
QUERY_CHECK_TARGET = 1

SIZES = {
    "AABB": 24, "INSTANCE": 72, "PRIMITIVE": 8, "MATERIAL": 84, "LIGHT": 40, "LIGHT_CONFIG": 52, "RESERVOIR": 36,
    "DI_INFO": 60, "VELOCITY": 8, "PATH_RESERVOIR": 92, "CAMERA_VIEW": 264, "STATUS": 96, "WORLD": 96, "RESTIR": 72,
    "RAY_QUERY": 40, "RAY_HIT": 16, "BRUSH_CONFIG": 28, "BRUSH_COUNTER": 8,
}

# feature bits (shared.inl:73-79)
TAA_BIT = 1 << 0
RIS_POINT_LIGHT_BIT = 1 << 1
RIS_ENV_LIGHT_BIT = 1 << 2
RIS_CUBE_LIGHT_BIT = 1 << 3
RIS_BRDF_BIT = 1 << 4
REMAP_BIT = 1 << 30

LIGHT_NONE, LIGHT_POINT, LIGHT_CUBE, LIGHT_ENV_MAP = 0, 1, 2, 5
MAX_INSTANCES = 983040
MAX_PRIMITIVES = 134217728
MAX_MATERIALS = 10000

# per-pixel state written by one frame (for the B_alg accounting and buffer sizing)
PER_PIXEL_BUFFERS = {
    "previous_reservoir": RESERVOIR, "intermediate_reservoir": RESERVOIR, "reservoir": RESERVOIR,
    "previous_di": DI_INFO, "di": DI_INFO, "velocity": VELOCITY, "output_path_reservoir": PATH_RESERVOIR,
    "temporal_path_reservoir": PATH_RESERVOIR, "indirect_color": np.dtype(("<f4", (3,))),
}



def view_buffer(key, raw):
    """Raw bytes of a per-pixel buffer as its records (vectors as (n, k))."""
    dt = PER_PIXEL_BUFFERS[key]
    raw = np.ascontiguousarray(raw).reshape(-1).view(np.uint8)
    if dt.subdtype is not None:
        base, shape = dt.subdtype
        return raw.view(base).reshape((-1,) + shape)
    return raw.view(dt)


for _n, _s in SIZES.items():
    assert globals()[_n].itemsize == _s, (_n, globals()[_n].itemsize, _s)
