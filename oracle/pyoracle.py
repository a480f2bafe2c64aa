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
# the same shader code built in double precision (Makefile, CT_ORACLE_FP64):
# every float of the structs and images is a double there
LIB64_PATH = os.path.join(HERE, "_ref", "libct_oracle64.so")
# FP32 built for the reference's own voxel edge (VOXEL_EXTENT 2^-5); the
# others are built for unit voxels
LIBE5_PATH = os.path.join(HERE, "_ref", "libct_oracle_e5.so")
E5 = 0.03125
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "cube-tracing_b200"))
from cube_tracing import layouts as L  # noqa: E402

_libs = {}


def lib_path(fp64=False, extent=1.0):
    if fp64:
        return LIB64_PATH
    return LIBE5_PATH if extent == E5 else LIB_PATH


def available(fp64=False, extent=1.0):
    return os.path.exists(lib_path(fp64, extent))


def lib(fp64=False, extent=1.0):
    path = lib_path(fp64, extent)
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run `make -C oracle`)")
        _lib = ctypes.CDLL(path)
        _libs[path] = _lib
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
        _lib.oracle_set_params.restype = ctypes.c_int
        _lib.oracle_set_params.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_intersect_box.restype = ctypes.c_int
        _lib.oracle_intersect_box.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return _libs[path]


# Flattened fields that open a nested struct holding a vector: in the FP64
# build that struct is 8-byte aligned.  PATH_RESERVOIR.rc_vertex_hit is an
# OBJECT_HIT {OBJECT_INFO object; vec3 hit;} (shared.inl).
_ALIGN8_GROUPS = {"rc_instance_id"}


def widen(dt):
    """The FP64 build's layout of a struct: every float32 a float64, fields
    in the same order at C alignment (the shim's vec3 is three doubles)."""
    dt = np.dtype(dt)
    if dt.names is None:
        if dt.subdtype is not None:
            base, shape = dt.subdtype
            return np.dtype((widen(base), shape))
        return np.dtype("<f8") if dt == np.dtype("<f4") else dt
    names, formats, offsets = [], [], []
    off, struct_align = 0, 1
    for n in dt.names:
        f = widen(dt.fields[n][0])
        a = max(f.alignment, 8 if n in _ALIGN8_GROUPS else 1)
        off = (off + a - 1) // a * a
        names.append(n)
        formats.append(f)
        offsets.append(off)
        off += f.itemsize
        struct_align = max(struct_align, a)
    size = (off + struct_align - 1) // struct_align * struct_align
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size})


class OracleInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "instance", "aabb", "primitive", "material", "light", "light_config", "reservoir", "di_info", "velocity",
        "path_reservoir", "camera_view", "status", "world", "restir", "push_constant")] + [("voxel_extent", ctypes.c_float)]


def info(fp64=False, extent=1.0):
    i = OracleInfo()
    lib(fp64, extent).oracle_info(ctypes.byref(i))
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


# The reuse parameters the oracle takes at run time (oracle_set_params), by
# their ct_params names, with the reference's compiled-in values
# (include/defines.glsl:34-62, compute/taa.glsl:13; one spatial round,
# rgen.glsl:394-397).
REFERENCE_PARAMS = {
    "min_ris_point_samples": 1, "max_ris_point_samples": 4, "min_ris_env_samples": 1, "max_ris_env_samples": 4,
    "min_ris_cube_samples": 4, "max_ris_cube_samples": 32, "min_num_of_neighbors": 3, "max_num_of_neighbors": 4,
    "pt_neighbor_count": 3, "pt_neighbor_radius": 1,
    "min_influence_from_the_past": 10.0, "max_influence_from_the_past": 20.0, "min_neighbors_radius": 2.0,
    "max_neighbors_radius": 50.0, "max_distance_to_hit": 1e3, "pt_max_influence_from_the_past": 20.0,
    "taa_alpha": 0.8, "spatial_passes": 1, "pt_shift_mapping": 0, "pt_near_field_distance": 0.0,
}
_PARAM_U = ["min_ris_point_samples", "max_ris_point_samples", "min_ris_env_samples", "max_ris_env_samples",
            "min_ris_cube_samples", "max_ris_cube_samples", "min_num_of_neighbors", "max_num_of_neighbors",
            "pt_neighbor_count", "pt_neighbor_radius", "pt_shift_mapping"]
_PARAM_F = ["min_influence_from_the_past", "max_influence_from_the_past", "min_neighbors_radius",
            "max_neighbors_radius", "max_distance_to_hit", "pt_max_influence_from_the_past", "taa_alpha",
            "pt_near_field_distance"]


def reuse_params(params=None):
    """REFERENCE_PARAMS updated from `params`: a mapping or an object with
    the ct_params field names (e.g. cube_tracing.native.Params); other
    fields are ignored."""
    out = dict(REFERENCE_PARAMS)
    if params is not None:
        for k in out:
            v = params.get(k) if isinstance(params, dict) else getattr(params, k, None)
            if v is not None:
                out[k] = v
    return out


class OracleRenderer:
    """Renders frames of a Scene on the host with the reference shaders."""

    def __init__(self, scene, width, height, threads=0, taa=True, features=L.RIS_CUBE_LIGHT_BIT, max_depth=3,
                 sky_time=1.0, is_afternoon=1, indirect=False, fp64=False, params=None):
        # fp64: the double-precision build of the same code; its buffers are
        # the widened layouts (widen) and its images float64
        # params: the run-time reuse parameters (reuse_params); the
        # reference's own values by default
        self.fp64 = fp64
        self.params = reuse_params(params)
        self._lib = lib(fp64, scene.voxel_extent)
        dt = widen if fp64 else np.dtype
        self._dt = dt
        built = info(fp64, scene.voxel_extent).voxel_extent
        if abs(built - scene.voxel_extent) > 0:
            raise ValueError(f"oracle built for VOXEL_EXTENT={built}, scene uses {scene.voxel_extent}")
        self.scene, self.W, self.H, self.threads = scene, width, height, threads
        self.taa, self.features = taa, features
        # indirect: rgen.glsl compiled with INDIRECT_ILLUMINATION_ON 1 (ReSTIR PT)
        self.indirect = indirect
        n = width * height
        self.buf = {k: np.zeros(n, dt(d)) for k, d in L.PER_PIXEL_BUFFERS.items()}
        fimg = np.float64 if fp64 else np.float32
        self.images = [np.zeros((height, width, 4), fimg) for _ in range(2)]
        self.taa_frame = np.zeros((height, width, 4), fimg)
        self.taa_prev = np.zeros((height, width, 4), fimg)
        self._imgs = {}
        self.world = np.zeros(1, L.WORLD)
        self._keep = [
            _nonempty(scene.instances, L.INSTANCE).astype(dt(L.INSTANCE)),
            _nonempty(scene.primitives, L.PRIMITIVE).astype(dt(L.PRIMITIVE)),
            _nonempty(scene.aabbs, L.AABB).astype(dt(L.AABB)), _nonempty(scene.materials, L.MATERIAL).astype(dt(L.MATERIAL)),
            _nonempty(scene.point_lights, L.LIGHT).astype(dt(L.LIGHT)),
            _nonempty(scene.cube_lights, L.LIGHT).astype(dt(L.LIGHT)),
            _nonempty(scene.env_lights, L.LIGHT).astype(dt(L.LIGHT)), np.zeros(max(scene.aabbs.shape[0], 1), np.uint32),
            np.zeros(max(scene.cube_lights.shape[0], 1), np.uint32)]
        inst, prim, aabb, mat, pl, cl, el, remap_p, remap_l = self._keep
        self.accel = self._lib.oracle_build_accel(_addr(inst), scene.instances.shape[0], _addr(aabb),
                                                  scene.aabbs.shape[0])
        if not self.accel:
            raise ValueError("scene AABBs are not grid-aligned voxels")
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
        self.restir = np.zeros(1, dt(L.RESTIR))
        # the same table with the current reservoirs bound as the
        # intermediate ones: the shading pass after an odd number of extra
        # spatial rounds reads them
        self.restir_swapped = np.zeros(1, dt(L.RESTIR))
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
        self.restir_swapped[0] = r
        self.restir_swapped[0]["intermediate_reservoir_address"] = _addr(self.buf["reservoir"])
        self.light_config = scene.light_config.astype(dt(L.LIGHT_CONFIG))
        self.camera = np.zeros(1, dt(L.CAMERA_VIEW))
        self.status = np.zeros(1, dt(L.STATUS))
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
                self._lib.oracle_free_accel(getattr(self, a))
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

    def apply_params(self):
        """Sets the library's run-time reuse parameters to this renderer's
        (they are process-wide; render() calls this before its passes)."""
        prm = self.params
        if not 1 <= int(prm["spatial_passes"]) <= 16:
            raise ValueError("spatial_passes must be in [1, 16]")
        u = np.array([prm[k] for k in _PARAM_U], np.uint32)
        f = np.array([prm[k] for k in _PARAM_F], np.float32)
        if self._lib.oracle_set_params(_addr(u), _addr(f)) != 0:
            raise ValueError("neighbour count above the oracle's capacity, or an unknown shift mapping")

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
        self.apply_params()
        n_rounds = int(self.params["spatial_passes"])
        for which in passes:
            if which == 3 and not taa_on:
                continue
            run_pc = pc
            if which == 2 and n_rounds > 1:
                # extra spatial rounds: intermediate -> current -> ..., then
                # the shading pass reads the last round's output
                for r in range(n_rounds - 1):
                    self._lib.oracle_pass(4 if r % 2 == 0 else 5, ctypes.byref(pc), self.threads, r0, r1)
                if (n_rounds - 1) % 2 == 1:
                    run_pc = self.push_constant()
                    run_pc.restir_buffer = _addr(self.restir_swapped)
            code = which + 10 if (self.indirect and which in (1, 2)) else which
            self._lib.oracle_pass(code, ctypes.byref(run_pc), self.threads, r0, r1)
        out = self.images[self.frame % 2]
        self.prev_cam = (np.array(inv_view), np.array(inv_proj))
        self.frame += 1
        if self.prev_accel:
            # the settling step after an edit: remap tables back to zero
            # (clear_instance_remapping_buffer, accel_struct_mngr.cpp:2616-2625)
            self._keep[7][:] = 0
            self._keep[8][:] = 0
            self._lib.oracle_free_accel(self.prev_accel)
            self.prev_accel = None
        return out

    # -- frame history checkpoint, in ct_state_save's blob format (include/ct.h)
    _STATE_SECTIONS = ["previous_reservoir", "intermediate_reservoir", "reservoir", "previous_di", "di", "velocity",
                       "output_path_reservoir", "temporal_path_reservoir", "indirect_color"]

    def _state_images(self, frame):
        cur, prev = self.images[frame % 2], self.images[(frame + 1) % 2]
        return [cur, prev if frame > 0 else cur, self.taa_frame, self.taa_prev]

    def save_state(self):
        """The history the last frame leaves for the next, as ct_state_save
        writes it, with the frame number and previous camera."""
        assert not self.fp64
        parts = [self.buf[k].view(np.uint8).reshape(-1) for k in self._STATE_SECTIONS]
        parts += [np.ascontiguousarray(im).view(np.uint8).reshape(-1) for im in self._state_images(self.frame - 1)]
        head = np.zeros(128, np.uint8)
        w = head.view(np.uint32)
        w[:6] = (0x54535443, 1, self.W, self.H, len(parts), 0)
        head[24:24 + 8 * len(parts)].view(np.uint64)[:] = [p.size for p in parts]
        return np.concatenate([head] + parts), self.frame, self.prev_cam

    def load_state(self, state):
        """Continues from a saved state (ct_state_save's blob, from either
        side): the next render() is the frame after the saved one.  The FP64
        build widens the single-precision records and images it loads (field
        by field, in order), so that it continues a CUDA or FP32 run from
        the same history."""
        blob, frame, prev_cam = state
        blob = np.ascontiguousarray(blob, np.uint8)
        w = blob[:24].view(np.uint32)
        if tuple(w[:5]) != (0x54535443, 1, self.W, self.H, 13):
            raise ValueError("not a saved state of this frame size")
        sizes = blob[24:24 + 8 * 13].view(np.uint64)
        off = 128
        n_px = self.W * self.H
        # single-precision record of each section (the images are RGBA32F)
        src_dt = [np.dtype(L.PER_PIXEL_BUFFERS[k]) for k in self._STATE_SECTIONS] + [np.dtype(("<f4", (4,)))] * 4
        dst = [self.buf[k] for k in self._STATE_SECTIONS] + list(self._state_images(frame - 1))
        for d, dt, n in zip(dst, src_dt, sizes):
            n = int(n)
            if n != n_px * dt.itemsize:
                raise ValueError("section size differs")
            part = blob[off:off + n]
            if not self.fp64:
                d.view(np.uint8).reshape(-1)[:] = part
            elif dt.names:
                d[:] = part.view(dt).astype(d.dtype)   # structured: by field position
            else:
                d[...] = part.view(np.float32).reshape(d.shape)
            off += n
        self.frame = frame
        self.prev_cam = prev_cam

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
            self._lib.oracle_free_accel(self.prev_accel)
        self._lib.oracle_accel_set_previous(self.accel, 1)
        self.prev_accel = self.accel
        self.accel = self._lib.oracle_build_accel(_addr(inst), inst.shape[0], _addr(aabb), aabb.shape[0])

    def queries(self, records, closest=False):
        """Runs ray queries (layouts.RAY_QUERY records) with the reference's
        is_vertex_visible / traceRayEXT on this renderer's scene."""
        records = np.ascontiguousarray(records, dtype=L.RAY_QUERY)
        n = records.shape[0]
        out = np.zeros(n, L.RAY_HIT) if closest else np.zeros(n, np.uint8)
        pc = self.push_constant()
        self._lib.oracle_queries(1 if closest else 0, ctypes.byref(pc), _addr(records), n, _addr(out), self.threads)
        return out

    @staticmethod
    def counters(reset=True):
        c = np.zeros(5, np.uint64)
        lib().oracle_counters(_addr(c), int(reset))
        return {"primary": int(c[0]), "shadow": int(c[1]), "bounce": int(c[2]), "voxel_tests": int(c[3]),
                "brick_visits": int(c[4])}


def precision_error(r32, r64, img32, img64, rows=None):
    """Error of a single-precision frame against the double-precision build
    of the same code on the same inputs (two OracleRenderer, fp64 False and
    True, after rendering the same frames): the share of hit pixels whose
    first-hit ids, final DI reservoir choice (Y, light type, seed, M) and,
    with PT, output path reservoir choice (flags, seeds, reconnection vertex,
    M) agree, and the relative error of the output image per pixel (largest
    channel, |x32 - x64| / max(|x64|, 1e-6)) as median, 99th percentile and
    maximum, over the pixels whose choices agree and over all pixels."""
    W, H = r32.W, r32.H
    r0, r1 = rows if rows is not None else (0, H)
    sel = slice(r0 * W, r1 * W)
    d32, d64 = r32.buf["di"][sel], r64.buf["di"][sel]
    hit = (d32["distance"] > 0) | (d64["distance"] > 0)
    ids = ((d32["distance"] > 0) == (d64["distance"] > 0)) & (d32["instance_id"] == d64["instance_id"]) & \
        (d32["primitive_id"] == d64["primitive_id"])
    q32, q64 = r32.buf["previous_reservoir"][sel], r64.buf["previous_reservoir"][sel]
    res = (q32["Y"] == q64["Y"]) & (q32["l_type"] == q64["l_type"]) & (q32["seed"] == q64["seed"]) & \
        (q32["M"] == q64["M"])
    paths = np.ones(res.shape, bool)
    if r32.indirect:
        p32, p64 = r32.buf["output_path_reservoir"][sel], r64.buf["output_path_reservoir"][sel]
        for k in ("path_flags", "rc_random_seed", "init_random_seed", "rc_instance_id", "rc_primitive_id", "M"):
            paths &= p32[k] == p64[k]
    a = np.asarray(img32[r0:r1, :, :3], np.float64)
    b = np.asarray(img64[r0:r1, :, :3], np.float64)
    rel = (np.abs(a - b) / np.maximum(np.abs(b), 1e-6)).max(-1).reshape(-1)
    same = ids & res & paths
    n = max(int(hit.sum()), 1)

    def stats(v):
        v = v if v.size else np.zeros(1)
        return {"median": float(np.median(v)), "p99": float(np.percentile(v, 99)), "max": float(v.max())}
    return {"pixels": int(rel.size), "hit_pixels": int(hit.sum()),
            "ids_equal": round(float((ids & hit).sum()) / n, 6),
            "reservoirs_equal": round(float((res & hit).sum()) / n, 6),
            "paths_equal": round(float((paths & hit).sum()) / n, 6),
            "image_rel_err": stats(rel[same]), "image_rel_err_all": stats(rel)}


def fpmath(x):
    """sin, cos and pow(x, 5) as the oracle's GLSL shim computes them."""
    x = np.ascontiguousarray(x, np.float32)
    s, c, p = np.empty_like(x), np.empty_like(x), np.empty_like(x)
    lib().oracle_fpmath(_addr(x), x.size, _addr(s), _addr(c), _addr(p))
    return s, c, p
