"""ctypes driver for the CPU parity oracle (oracle/_ref/libct_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the product package.

It renders frames with the reference's own shader code (see
oracle/oracle_main.cpp) on host buffers laid out like the GPU path's, in the
order App::draw records the passes (src/main.cpp:1436-1703): pass 1
(rgen.glsl RESTIR_PREPASS_AND_FIRST_VISIBILITY_TEST), pass 2
(THIRD_VISIBILITY_TEST_AND_SHADING_PASS), then TAA when the frame has a
previous image (main.cpp:1483-1487), after which the output images swap.
With `indirect=True` both ray-generation passes run with the ReSTIR PT
blocks compiled in (INDIRECT_ILLUMINATION_ON 1).
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libct_oracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "cube-tracing_b200"))
from cube_tracing import layouts as L  # noqa: E402

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_build_accel.restype = ctypes.c_void_p
        _lib.oracle_build_accel.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32]
        _lib.oracle_free_accel.argtypes = [ctypes.c_void_p]
        _lib.oracle_accel_set_previous.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _lib.oracle_pass.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
        _lib.oracle_counters.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _lib.oracle_tea.restype = ctypes.c_uint32
        _lib.oracle_tea.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib.oracle_rnd.restype = ctypes.c_float
        _lib.oracle_rnd.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
        _lib.oracle_compute_ray_origin.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_queries.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                        ctypes.c_void_p, ctypes.c_int]
        _lib.oracle_fpmath.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
        _lib.oracle_intersect_box.restype = ctypes.c_int
        _lib.oracle_intersect_box.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return _lib


class OracleInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "instance", "aabb", "primitive", "material", "light", "light_config", "reservoir", "di_info", "velocity",
        "path_reservoir", "camera_view", "status", "world", "restir", "push_constant")] + [("voxel_extent", ctypes.c_float)]


def info():
    i = OracleInfo()
    lib().oracle_info(ctypes.byref(i))
    return i


class GlslImage(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("texels", ctypes.c_void_p)]


class PushConstant(ctypes.Structure):
    _fields_ = [("size", ctypes.c_uint32 * 2), ("tlas", ctypes.c_void_p), ("tlas_previous", ctypes.c_void_p),
                ("swapchain", ctypes.c_void_p), ("previous_swapchain", ctypes.c_void_p),
                ("taa_frame", ctypes.c_void_p), ("taa_prev_frame", ctypes.c_void_p),
                ("camera_buffer", ctypes.c_void_p), ("status_buffer", ctypes.c_void_p),
                ("world_buffer", ctypes.c_void_p), ("restir_buffer", ctypes.c_void_p)]


def _addr(a):
    return a.ctypes.data


def _nonempty(a, dtype):
    return a if a.shape[0] > 0 else np.zeros(1, dtype)


class OracleRenderer:
    """Renders frames of a Scene on the host with the reference shaders."""

    def __init__(self, scene, width, height, threads=0, taa=True, features=L.RIS_CUBE_LIGHT_BIT, max_depth=3,
                 sky_time=1.0, is_afternoon=1, indirect=False):
        if abs(info().voxel_extent - scene.voxel_extent) > 0:
            raise ValueError(f"oracle built for VOXEL_EXTENT={info().voxel_extent}, scene uses {scene.voxel_extent}")
        self.scene, self.W, self.H, self.threads = scene, width, height, threads
        self.taa, self.features = taa, features
        # indirect: rgen.glsl compiled with INDIRECT_ILLUMINATION_ON 1 (ReSTIR PT)
        self.indirect = indirect
        self.accel = lib().oracle_build_accel(_addr(scene.instances), scene.instances.shape[0], _addr(scene.aabbs),
                                              scene.aabbs.shape[0])
        if not self.accel:
            raise ValueError("scene AABBs are not grid-aligned voxels")
        n = width * height
        self.buf = {k: np.zeros(n, dt) for k, dt in L.PER_PIXEL_BUFFERS.items()}
        self.images = [np.zeros((height, width, 4), np.float32) for _ in range(2)]
        self.taa_frame = np.zeros((height, width, 4), np.float32)
        self.taa_prev = np.zeros((height, width, 4), np.float32)
        self._imgs = {}
        self.world = np.zeros(1, L.WORLD)
        self._keep = [
            _nonempty(scene.instances, L.INSTANCE), _nonempty(scene.primitives, L.PRIMITIVE),
            _nonempty(scene.aabbs, L.AABB), _nonempty(scene.materials, L.MATERIAL),
            _nonempty(scene.point_lights, L.LIGHT), _nonempty(scene.cube_lights, L.LIGHT),
            _nonempty(scene.env_lights, L.LIGHT), np.zeros(max(scene.aabbs.shape[0], 1), np.uint32),
            np.zeros(max(scene.cube_lights.shape[0], 1), np.uint32)]
        inst, prim, aabb, mat, pl, cl, el, remap_p, remap_l = self._keep
        w = self.world[0]
        w["instance_address"] = w["instance_address_prev"] = _addr(inst)
        w["primitive_address"] = w["primitive_address_prev"] = _addr(prim)
        w["aabb_address"] = w["aabb_address_prev"] = _addr(aabb)
        w["remapped_primitive_address"] = _addr(remap_p)
        w["remapped_cube_light_address"] = _addr(remap_l)
        w["material_address"] = _addr(mat)
        w["point_light_address"] = _addr(pl)
        w["cube_light_address"] = _addr(cl)
        w["env_light_address"] = _addr(el)
        self.restir = np.zeros(1, L.RESTIR)
        r = self.restir[0]
        r["previous_reservoir_address"] = _addr(self.buf["previous_reservoir"])
        r["intermediate_reservoir_address"] = _addr(self.buf["intermediate_reservoir"])
        r["reservoir_address"] = _addr(self.buf["reservoir"])
        r["previous_di_address"] = _addr(self.buf["previous_di"])
        r["di_address"] = _addr(self.buf["di"])
        r["velocity_address"] = _addr(self.buf["velocity"])
        r["output_path_reservoir_address"] = _addr(self.buf["output_path_reservoir"])
        r["temporal_path_reservoir_address"] = _addr(self.buf["temporal_path_reservoir"])
        r["indirect_color_address"] = _addr(self.buf["indirect_color"])
        self.light_config = scene.light_config.copy()
        self.camera = np.zeros(1, L.CAMERA_VIEW)
        self.status = np.zeros(1, L.STATUS)
        s = self.status[0]
        s["resolution"] = (width, height)
        s["light_config_address"] = _addr(self.light_config)
        s["obj_count"] = scene.aabbs.shape[0]
        s["time"] = sky_time
        s["is_afternoon"] = is_afternoon
        s["max_depth"] = max_depth
        self.frame = 0
        self.prev_cam = None
        # scene before the last edit, bound as tlas_previous for one frame
        self.prev_accel = None

    def close(self):
        for a in ("accel", "prev_accel"):
            if getattr(self, a, None):
                lib().oracle_free_accel(getattr(self, a))
                setattr(self, a, None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _img(self, a):
        key = id(a)
        if key not in self._imgs:
            self._imgs[key] = (GlslImage(self.W, self.H, _addr(a)), a)
        return ctypes.addressof(self._imgs[key][0])

    def push_constant(self):
        cur, prev = self.images[self.frame % 2], self.images[(self.frame + 1) % 2]
        pc = PushConstant()
        pc.size[0], pc.size[1] = self.W, self.H
        pc.tlas = self.accel
        pc.tlas_previous = self.prev_accel if self.prev_accel else self.accel
        pc.swapchain = self._img(cur)
        pc.previous_swapchain = self._img(prev if self.frame > 0 else cur)
        pc.taa_frame = self._img(self.taa_frame)
        pc.taa_prev_frame = self._img(self.taa_prev)
        pc.camera_buffer = _addr(self.camera)
        pc.status_buffer = _addr(self.status)
        pc.world_buffer = _addr(self.world)
        pc.restir_buffer = _addr(self.restir)
        return pc

    def set_time(self, time, is_afternoon):
        s = self.status[0]
        s["time"] = time
        s["is_afternoon"] = int(bool(is_afternoon))

    def set_point_lights(self, lights):
        """Overwrites the scene's point lights in place (the buffer WORLD points at)."""
        self._keep[4][:] = lights

    def set_camera(self, inv_view, inv_proj):
        c = self.camera[0]
        c["inv_view"], c["inv_proj"] = inv_view, inv_proj
        pv, pp = self.prev_cam if self.prev_cam is not None else (inv_view, inv_proj)
        c["prev_inv_view"], c["prev_inv_proj"] = pv, pp

    def render(self, inv_view, inv_proj, passes=(1, 2, 3), rows=None):
        """One frame.  Returns the output image (H, W, 4)."""
        self.set_camera(inv_view, inv_proj)
        taa_on = self.taa and self.frame > 0
        self.status[0]["frame_number"] = self.frame
        remap = L.REMAP_BIT if self.prev_accel else 0
        self.status[0]["is_active"] = self.features | (L.TAA_BIT if taa_on else 0) | remap
        pc = self.push_constant()
        r0, r1 = rows if rows is not None else (0, 0)
        for which in passes:
            if which == 3 and not taa_on:
                continue
            code = which + 10 if (self.indirect and which in (1, 2)) else which
            lib().oracle_pass(code, ctypes.byref(pc), self.threads, r0, r1)
        out = self.images[self.frame % 2]
        self.prev_cam = (np.array(inv_view), np.array(inv_proj))
        self.frame += 1
        if self.prev_accel:
            # the settling step after an edit: remap tables back to zero
            # (clear_instance_remapping_buffer, accel_struct_mngr.cpp:2616-2625)
            self._keep[7][:] = 0
            self._keep[8][:] = 0
            lib().oracle_free_accel(self.prev_accel)
            self.prev_accel = None
        return out

    def erase(self, pixel, window):
        """Brush + rearrangement (oracle/edits.py) at `pixel` of the last
        frame with a square window of half width `window`, then a rebuild;
        the next frame renders with REMAP_BIT and the old scene as
        tlas_previous.  Returns (marked primitives, marked instances)."""
        import edits
        marks = edits.brush(self.buf["previous_di"], self.W, self.H, pixel, window, self._keep[0])
        self.remove(marks[0], marks[1])
        return marks

    def remove(self, marked_prims, marked_insts):
        """Rearrangement (oracle/edits.py) of the given global primitives of
        the given instances, then a rebuild; the next frame renders with
        REMAP_BIT and the old scene as tlas_previous."""
        import edits
        inst, prim, aabb, mat, pl, cl, el, remap_p, remap_l = self._keep
        edits.rearrange(inst, prim, aabb, cl, self.light_config, marked_prims, marked_insts, remap_p, remap_l)
        if self.prev_accel:
            lib().oracle_free_accel(self.prev_accel)
        lib().oracle_accel_set_previous(self.accel, 1)
        self.prev_accel = self.accel
        self.accel = lib().oracle_build_accel(_addr(inst), inst.shape[0], _addr(aabb), aabb.shape[0])

    def queries(self, records, closest=False):
        """Runs ray queries (layouts.RAY_QUERY records) with the reference's
        is_vertex_visible / traceRayEXT on this renderer's scene."""
        records = np.ascontiguousarray(records, dtype=L.RAY_QUERY)
        n = records.shape[0]
        out = np.zeros(n, L.RAY_HIT) if closest else np.zeros(n, np.uint8)
        pc = self.push_constant()
        lib().oracle_queries(1 if closest else 0, ctypes.byref(pc), _addr(records), n, _addr(out), self.threads)
        return out

    @staticmethod
    def counters(reset=True):
        c = np.zeros(5, np.uint64)
        lib().oracle_counters(_addr(c), int(reset))
        return {"primary": int(c[0]), "shadow": int(c[1]), "bounce": int(c[2]), "voxel_tests": int(c[3]),
                "brick_visits": int(c[4])}


def fpmath(x):
    """sin, cos and pow(x, 5) as the oracle's GLSL shim computes them."""
    x = np.ascontiguousarray(x, np.float32)
    s, c, p = np.empty_like(x), np.empty_like(x), np.empty_like(x)
    lib().oracle_fpmath(_addr(x), x.size, _addr(s), _addr(c), _addr(p))
    return s, c, p
