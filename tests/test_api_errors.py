"""Host-side argument checking of the C ABI.  Every case here is rejected
before any CUDA call, so it runs without a GPU."""
import ctypes

import pytest

from cube_tracing import native


def call(name, *args):
    return getattr(native.lib(), name)(*args)


def test_null_arguments_rejected():
    assert call("ct_build_accel", None, None, None) == 1
    assert call("ct_accel_free", None) == 1
    assert call("ct_accel_get_info", None, None) == 1
    g, c = (ctypes.c_int32 * 3)(), (ctypes.c_uint32 * 3)()
    assert call("ct_accel_field", None, 0, 0, None, ctypes.byref(g), ctypes.byref(c), None) == 1
    assert call("ct_trace_frame", None, None, None) == 1
    assert call("ct_get_error", None, 0, None) == 1


def test_scene_description_checked():
    h = ctypes.c_void_p()
    d = native.SceneDesc(0, 1, 0, 0, 1, 1.0)
    assert call("ct_build_accel", ctypes.byref(d), ctypes.byref(h), None) == 1
    d = native.SceneDesc(256, 0, 0, 512, 1, 1.0)     # no instances
    assert call("ct_build_accel", ctypes.byref(d), ctypes.byref(h), None) == 1
    d = native.SceneDesc(256, 1, 0, 512, 1, float("nan"))
    assert call("ct_build_accel", ctypes.byref(d), ctypes.byref(h), None) == 1
    d = native.SceneDesc(256, 1, 0, 512, 1, -1.0)
    assert call("ct_build_accel", ctypes.byref(d), ctypes.byref(h), None) == 1
    d = native.SceneDesc(256, 10 ** 6, 0, 512, 1, 1.0)  # above MAX_INSTANCES
    assert call("ct_build_accel", ctypes.byref(d), ctypes.byref(h), None) == 2
    d = native.SceneDesc(258, 1, 0, 512, 1, 1.0)     # misaligned INSTANCE buffer
    assert call("ct_build_accel", ctypes.byref(d), ctypes.byref(h), None) == 1
    assert h.value is None


def valid_pc():
    pc = native.PushConstant()
    pc.size[0], pc.size[1] = 64, 64
    # never dereferenced: every case below fails an earlier check
    pc.tlas = pc.tlas_previous = 1 << 20
    pc.swapchain = pc.previous_swapchain = pc.taa_frame = pc.taa_prev_frame = 4096
    pc.camera_buffer = pc.status_buffer = pc.world_buffer = pc.restir_buffer = 8192
    return pc


@pytest.mark.parametrize("mutate, expect", [
    (lambda pc, p: setattr(pc, "tlas", None), 1),                     # no acceleration structure
    (lambda pc, p: pc.size.__setitem__(0, 0), 1),                     # empty frame
    (lambda pc, p: setattr(pc, "camera_buffer", 0), 1),
    (lambda pc, p: setattr(pc, "swapchain", 4100), 1),                # image not 16-byte aligned
    (lambda pc, p: setattr(p, "struct_size", 3), 1),                  # wrong params version
    (lambda pc, p: setattr(p, "max_num_of_neighbors", 9), 2),         # above CT_MAX_NEIGHBORS
    (lambda pc, p: setattr(p, "spatial_passes", 0), 1),
    (lambda pc, p: setattr(p, "taa_alpha", float("inf")), 5),
    (lambda pc, p: setattr(p, "walk_step_limit", (1 << 16) + 1), 1),  # above the built-in walk cap
])
def test_frame_arguments_checked(mutate, expect):
    pc, p = valid_pc(), native.default_params()
    mutate(pc, p)
    assert call("ct_trace_frame", ctypes.byref(pc), ctypes.byref(p), None) == expect
    assert call("ct_restir_di", ctypes.byref(pc), ctypes.byref(p), 0, None) == expect


def test_taa_checks_without_accel():
    pc, p = valid_pc(), native.default_params()
    p.max_num_of_neighbors = 9
    assert call("ct_taa", ctypes.byref(pc), ctypes.byref(p), None) == 2
    p = native.default_params()
    pc.previous_swapchain = 0
    assert call("ct_taa", ctypes.byref(pc), ctypes.byref(p), None) == 1




def test_counter_flag_requires_buffer():
    pc, p = valid_pc(), native.default_params()
    p.flags = native.CT_PARAM_COUNT_RAYS
    p.counters_address = 0
    assert call("ct_taa", ctypes.byref(pc), ctypes.byref(p), None) == 1
