"""ctypes binding of libct.so (include/ct.h).

The library is the product: every call goes to the CUDA kernels.  There is
no fallback; if libct.so is missing or fails to load, importing this module
raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libct.so")

CT_OK = 0
STATUS_NAMES = {0: "CT_OK", 1: "CT_ERR_INVALID_ARG", 2: "CT_ERR_CAPACITY", 3: "CT_ERR_CUDA", 4: "CT_ERR_ITER_LIMIT",
                5: "CT_ERR_NAN_INPUT", 6: "CT_ERR_UNSUPPORTED", 7: "CT_ERR_NOT_GRID_ALIGNED"}
CT_PARAM_COUNT_RAYS = 1
CT_PARAM_INDIRECT = 2
CT_SHIFT_RECONNECTION = 0
CT_SHIFT_HYBRID = 2
CT_MAX_NEIGHBORS = 8


class CtError(RuntimeError):
    def __init__(self, fn, status, detail=""):
        self.status = status
        super().__init__(f"{fn} failed: {STATUS_NAMES.get(status, status)} {detail}".strip())


class PushConstant(ctypes.Structure):
    _fields_ = [("size", ctypes.c_uint32 * 2), ("tlas", ctypes.c_void_p), ("tlas_previous", ctypes.c_void_p),
                ("swapchain", ctypes.c_void_p), ("previous_swapchain", ctypes.c_void_p),
                ("taa_frame", ctypes.c_void_p), ("taa_prev_frame", ctypes.c_void_p),
                ("camera_buffer", ctypes.c_uint64), ("status_buffer", ctypes.c_uint64),
                ("world_buffer", ctypes.c_uint64), ("restir_buffer", ctypes.c_uint64)]


class Params(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("voxel_extent", ctypes.c_float),
                ("min_ris_point_samples", ctypes.c_uint32), ("max_ris_point_samples", ctypes.c_uint32),
                ("min_ris_env_samples", ctypes.c_uint32), ("max_ris_env_samples", ctypes.c_uint32),
                ("min_ris_cube_samples", ctypes.c_uint32), ("max_ris_cube_samples", ctypes.c_uint32),
                ("min_influence_from_the_past", ctypes.c_float), ("max_influence_from_the_past", ctypes.c_float),
                ("min_num_of_neighbors", ctypes.c_uint32), ("max_num_of_neighbors", ctypes.c_uint32),
                ("min_neighbors_radius", ctypes.c_float), ("max_neighbors_radius", ctypes.c_float),
                ("max_distance_to_hit", ctypes.c_float), ("spatial_passes", ctypes.c_uint32),
                ("taa_alpha", ctypes.c_float), ("flags", ctypes.c_uint32), ("pt_neighbor_count", ctypes.c_uint32),
                ("pt_neighbor_radius", ctypes.c_int32), ("pt_max_influence_from_the_past", ctypes.c_float),
                ("walk_step_limit", ctypes.c_uint32), ("counters_address", ctypes.c_uint64),
                ("workspace_address", ctypes.c_uint64), ("workspace_bytes", ctypes.c_uint64),
                ("walker_blocks", ctypes.c_uint32), ("pt_shift_mapping", ctypes.c_uint32),
                ("pt_near_field_distance", ctypes.c_float), ("_reserved", ctypes.c_uint32)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("instance_address", ctypes.c_uint64), ("instance_count", ctypes.c_uint32), ("_pad", ctypes.c_uint32),
                ("aabb_address", ctypes.c_uint64), ("aabb_count", ctypes.c_uint32), ("voxel_extent", ctypes.c_float)]


class AccelInfo(ctypes.Structure):
    _fields_ = [("instance_count", ctypes.c_uint32), ("brick_count", ctypes.c_uint32), ("voxel_count", ctypes.c_uint32),
                ("grid_exact", ctypes.c_uint32), ("device_bytes", ctypes.c_uint64), ("grid_min", ctypes.c_int32 * 3),
                ("grid_dim", ctypes.c_int32 * 3)]


class ErrorInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("detail", ctypes.c_uint32), ("pixel", ctypes.c_uint32),
                ("_pad", ctypes.c_uint32)]


class View(ctypes.Structure):
    _fields_ = [("pc", PushConstant), ("params", Params), ("is_active", ctypes.c_uint32), ("lane", ctypes.c_uint32)]


CT_MAX_LANES = 64


class AdjointDesc(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("spp", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("seed", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("primitive_count", ctypes.c_uint32), ("emitter_count", ctypes.c_uint32),
                ("rect", ctypes.c_uint32 * 4), ("miss_radiance", ctypes.c_float), ("camera_address", ctypes.c_uint64),
                ("emitter_index_address", ctypes.c_uint64)]


class NrcFrame(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("train_paths", ctypes.c_uint32), ("train_offset", ctypes.c_uint32),
                ("train_bounces", ctypes.c_uint32), ("cache_vertex", ctypes.c_uint32), ("_reserved", ctypes.c_uint32),
                ("base_address", ctypes.c_uint64),
                ("query_address", ctypes.c_uint64), ("throughput_address", ctypes.c_uint64),
                ("train_query_address", ctypes.c_uint64), ("train_partial_address", ctypes.c_uint64),
                ("train_throughput_address", ctypes.c_uint64)]


CT_ADJOINT_IMAGE_F64 = 1
CT_ADJOINT_MAX_DEPTH = 16


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("total_ms", ctypes.c_double), ("launches", ctypes.c_uint64)]


# exported entry points and their signatures (include/ct.h)
_SIGS = {
    "ct_abi_version": (ctypes.c_uint32, []),
    "ct_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "ct_last_cuda_error": (ctypes.c_char_p, []),
    "ct_params_default": (None, [ctypes.POINTER(Params)]),
    "ct_build_accel": (ctypes.c_int, [ctypes.POINTER(SceneDesc), ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    "ct_accel_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AccelInfo)]),
    "ct_accel_free": (ctypes.c_int, [ctypes.c_void_p]),
    "ct_accel_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_int32 * 3), ctypes.POINTER(ctypes.c_uint32 * 3),
                                      ctypes.c_void_p]),
    "ct_trace_frame": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.POINTER(Params), ctypes.c_void_p]),
    "ct_restir_di": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.POINTER(Params), ctypes.c_int,
                                     ctypes.c_void_p]),
    "ct_restir_di_static": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.POINTER(Params), ctypes.c_int,
                                           ctypes.c_void_p]),
    "ct_restir_pt": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.POINTER(Params), ctypes.c_int,
                                    ctypes.c_void_p]),
    "ct_taa": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.POINTER(Params), ctypes.c_void_p]),
    "ct_render_frame": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.POINTER(Params), ctypes.c_uint32,
                                        ctypes.c_void_p]),
    "ct_get_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ErrorInfo)]),
    "ct_trace_visibility": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "ct_trace_closest": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "ct_brush": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.c_void_p]),
    "ct_rearrange": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]),
    "ct_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "ct_profile_read": (ctypes.c_int, [ctypes.POINTER(KernelTime), ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.c_int]),
    "ct_workspace_size": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(Params),
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "ct_render_views": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32,
                                       ctypes.c_void_p]),
    "ct_nrc_encode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "ct_nrc_infer": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                    ctypes.c_void_p]),
    "ct_nrc_infer_encoded": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "ct_nrc_status": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p]),
    "ct_nrc_trace": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p]),
    "ct_adjoint_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdjointDesc), ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ct_adjoint_backward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AdjointDesc), ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "ct_state_size": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]),
    "ct_state_save": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "ct_state_load": (ctypes.c_int, [ctypes.POINTER(PushConstant), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
}

# ct_state_save blob (include/ct.h): header, then these sections in order
STATE_MAGIC = 0x54535443
STATE_VERSION = 1
STATE_HEADER_BYTES = 128
STATE_SECTIONS = ["previous_reservoir", "intermediate_reservoir", "reservoir", "previous_di", "di", "velocity",
                  "output_path_reservoir", "temporal_path_reservoir", "indirect_color", "swapchain",
                  "previous_swapchain", "taa_frame", "taa_prev_frame"]

_lib = None


def lib():
    """The loaded libct.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libct.so not built: {LIB_PATH} (run python cube-tracing_b200/build.py)")
        _lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(fn_name, status):
    if status != CT_OK:
        detail = ""
        if status == 3:
            detail = lib().ct_last_cuda_error().decode()
        raise CtError(fn_name, status, detail)


def default_params(**overrides):
    p = Params()
    lib().ct_params_default(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def params_for_scene(scene, **overrides):
    return default_params(voxel_extent=scene.voxel_extent, **overrides)


def params_dict(p):
    return {name: getattr(p, name) for name, _ in Params._fields_}


def kernel_times(reset=True):
    """{kernel name: (total ms, launches)} recorded since the last reset
    (needs ct_profile_enable(1))."""
    buf = (KernelTime * 32)()
    n = ctypes.c_uint32()
    check("ct_profile_read", lib().ct_profile_read(buf, 32, ctypes.byref(n), int(reset)))
    return {buf[i].name.decode(): (buf[i].total_ms, int(buf[i].launches)) for i in range(min(n.value, 32))}
