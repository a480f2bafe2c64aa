"""Frame driver: owns the device buffers of one view and records a frame the
way cube-tracing's App::draw does (src/main.cpp:1436-1703).

  * camera and Status blocks are uploaded from host copies each frame
    (main.cpp:1450-1556); the previous frame's matrices become prev_*
    (main.cpp:1660-1666);
  * pass 1 (ct_trace_frame + ct_restir_di stage 0), pass 2 (ct_restir_di
    stage 1), then TAA when there is a previous output image and filtering
    is on (main.cpp:1483-1487, 1617-1651);
  * two output images alternate: this frame's output is the next frame's
    previous_swapchain.

Device memory comes from torch's caching allocator; the kernels run on the
current torch CUDA stream.  Host arrays use the layouts of `layouts.py`.
"""
import ctypes

import numpy as np
import torch

from . import layouts as L
from . import native


def _dev(arr, device):
    a = np.ascontiguousarray(arr)
    if a.nbytes == 0:
        a = np.zeros(1, a.dtype)
    return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(device)


class Accel:
    """ct_build_accel over a scene's instance and AABB buffers on the device."""

    def __init__(self, instances_dev, n_inst, aabbs_dev, n_aabb, voxel_extent, stream=None):
        desc = native.SceneDesc(instances_dev.data_ptr(), n_inst, 0, aabbs_dev.data_ptr(), n_aabb, voxel_extent)
        h = ctypes.c_void_p()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        native.check("ct_build_accel", native.lib().ct_build_accel(ctypes.byref(desc), ctypes.byref(h), s))
        self.handle = h.value

    def info(self):
        i = native.AccelInfo()
        native.check("ct_accel_get_info", native.lib().ct_accel_get_info(self.handle, ctypes.byref(i)))
        return i

    def field(self, instance=0, octant=0):
        """The walk's cell field of one grid and ray octant (ct_accel_field):
        (edges as a uint8 array [z, y, x], the grid's first voxel coordinate)."""
        gmin, cells = (ctypes.c_int32 * 3)(), (ctypes.c_uint32 * 3)()
        lib = native.lib()
        native.check("ct_accel_field", lib.ct_accel_field(self.handle, instance, octant, None, ctypes.byref(gmin),
                                                          ctypes.byref(cells), None))
        X, Y, Z = cells
        out = torch.empty((Z, Y, X), dtype=torch.uint8, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        native.check("ct_accel_field", lib.ct_accel_field(self.handle, instance, octant, out.data_ptr(),
                                                          ctypes.byref(gmin), ctypes.byref(cells), s))
        return out.cpu().numpy(), tuple(gmin)

    def free(self):
        if self.handle:
            native.lib().ct_accel_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class SceneBuffers:
    """The scene's WORLD-table buffers on the device and the acceleration
    structure built from them."""

    def __init__(self, scene, device="cuda"):
        self.scene = scene
        self.device = device
        self.instances = _dev(scene.instances, device)
        self.primitives = _dev(scene.primitives, device)
        self.aabbs = _dev(scene.aabbs, device)
        self.materials = _dev(scene.materials, device)
        self.point_lights = _dev(scene.point_lights, device)
        self.cube_lights = _dev(scene.cube_lights, device)
        self.env_lights = _dev(scene.env_lights, device)
        self.n_instances, self.n_primitives = scene.instances.shape[0], scene.aabbs.shape[0]
        # scene edits (ct_brush / ct_rearrange): remap tables, brush bitmasks and counter
        self.remap_p = torch.zeros(max(self.n_primitives, 1), dtype=torch.int32, device=device)
        self.remap_l = torch.zeros(max(scene.cube_lights.shape[0], 1), dtype=torch.int32, device=device)
        self.primitive_bitmask = torch.zeros((self.n_primitives + 31) // 32 + 1, dtype=torch.int32, device=device)
        self.instance_bitmask = torch.zeros((self.n_instances + 31) // 32 + 1, dtype=torch.int32, device=device)
        self.brush_counter = torch.zeros(2, dtype=torch.int32, device=device)
        self.brush_config = torch.zeros(L.BRUSH_CONFIG.itemsize, dtype=torch.uint8, device=device)
        self.light_config = _dev(scene.light_config, device)
        self.accel = Accel(self.instances, self.n_instances, self.aabbs, self.n_primitives, scene.voxel_extent)
        # the structure before the last edit, bound as tlas_previous for one
        # frame, then kept until the next edit
        self.accel_prev = None
        self.accel_retired = []
        w = np.zeros(1, L.WORLD)[0]
        w["instance_address"] = w["instance_address_prev"] = self.instances.data_ptr()
        w["primitive_address"] = w["primitive_address_prev"] = self.primitives.data_ptr()
        w["aabb_address"] = w["aabb_address_prev"] = self.aabbs.data_ptr()
        w["remapped_primitive_address"] = self.remap_p.data_ptr()
        w["remapped_cube_light_address"] = self.remap_l.data_ptr()
        w["material_address"] = self.materials.data_ptr()
        w["point_light_address"] = self.point_lights.data_ptr()
        w["cube_light_address"] = self.cube_lights.data_ptr()
        w["env_light_address"] = self.env_lights.data_ptr()
        self.world = _dev(np.array([w], L.WORLD), device)

    def set_point_lights(self, lights):
        """Overwrites the point-light buffer (same count), e.g. the moving sun
        of cube_tracing.daylight."""
        lights = np.ascontiguousarray(lights, L.LIGHT)
        if lights.shape[0] * L.LIGHT.itemsize != self.point_lights.numel():
            raise ValueError("point light count differs from the scene's")
        self.point_lights.copy_(torch.from_numpy(lights.view(np.uint8).copy()).to(self.point_lights.device))


class Renderer:
    """One view of a scene: per-pixel ReSTIR buffers, images and the frame loop."""

    def __init__(self, scene, width, height, params=None, taa=True, features=L.RIS_CUBE_LIGHT_BIT, max_depth=3,
                 sky_time=1.0, is_afternoon=1, device="cuda", scene_buffers=None, count_rays=False, indirect=False):
        self.sb = scene_buffers if scene_buffers is not None else SceneBuffers(scene, device)
        self.scene, self.W, self.H, self.device = scene, width, height, device
        # params: a native.Params, or a mapping of ct_params field overrides
        # applied to the scene's defaults
        if params is None:
            params = native.params_for_scene(scene)
        elif isinstance(params, dict):
            params = native.params_for_scene(scene, **params)
        self.params = params
        self.taa, self.features = taa, features
        n = width * height
        self.buf = {k: torch.zeros(n * dt.itemsize, dtype=torch.uint8, device=device)
                    for k, dt in L.PER_PIXEL_BUFFERS.items()}
        self.images = [torch.zeros((height, width, 4), dtype=torch.float32, device=device) for _ in range(2)]
        self.taa_frame = torch.zeros((height, width, 4), dtype=torch.float32, device=device)
        self.taa_prev = torch.zeros((height, width, 4), dtype=torch.float32, device=device)
        r = np.zeros(1, L.RESTIR)[0]
        for field, key in (("previous_reservoir_address", "previous_reservoir"),
                           ("intermediate_reservoir_address", "intermediate_reservoir"),
                           ("reservoir_address", "reservoir"), ("previous_di_address", "previous_di"),
                           ("di_address", "di"), ("velocity_address", "velocity"),
                           ("output_path_reservoir_address", "output_path_reservoir"),
                           ("temporal_path_reservoir_address", "temporal_path_reservoir"),
                           ("indirect_color_address", "indirect_color")):
            r[field] = self.buf[key].data_ptr()
        self.restir = _dev(np.array([r], L.RESTIR), device)
        self.status_host = np.zeros(1, L.STATUS)
        s = self.status_host[0]
        s["resolution"] = (width, height)
        s["light_config_address"] = self.sb.light_config.data_ptr()
        s["obj_count"] = scene.aabbs.shape[0]
        s["time"] = sky_time
        s["is_afternoon"] = is_afternoon
        s["max_depth"] = max_depth
        s["brush_config_address"] = self.sb.brush_config.data_ptr()
        s["brush_counter_address"] = self.sb.brush_counter.data_ptr()
        s["instance_bitmask_address"] = self.sb.instance_bitmask.data_ptr()
        s["primitive_bitmask_address"] = self.sb.primitive_bitmask.data_ptr()
        self.status = torch.zeros(L.STATUS.itemsize, dtype=torch.uint8, device=device)
        self.camera_host = np.zeros(1, L.CAMERA_VIEW)
        self.camera = torch.zeros(L.CAMERA_VIEW.itemsize, dtype=torch.uint8, device=device)
        # pinned staging ring for the per-frame uploads; a slot is reused only
        # after the copy that last read it has completed
        self._ring = [(torch.zeros(L.CAMERA_VIEW.itemsize + L.STATUS.itemsize, dtype=torch.uint8).pin_memory(),
                       torch.cuda.Event()) for _ in range(8)]
        self._ring_pos = 0
        self._ring_used = [False] * len(self._ring)
        self.counters = torch.zeros(16, dtype=torch.int64, device=device)
        # indirect: the ReSTIR PT stages run (INDIRECT_ILLUMINATION_ON)
        if indirect:
            self.params.flags |= native.CT_PARAM_INDIRECT
        if count_rays:
            self.params.flags |= native.CT_PARAM_COUNT_RAYS
            self.params.counters_address = self.counters.data_ptr()
        # the view's own scratch (ct_params.workspace_address), so that an
        # edit's rebuilt acceleration structure needs none of its own
        need = ctypes.c_uint64()
        native.check("ct_workspace_size", native.lib().ct_workspace_size(width, height, ctypes.byref(self.params),
                                                                         ctypes.byref(need)))
        self.workspace = torch.empty(need.value + 256, dtype=torch.uint8, device=device)
        self.params.workspace_address = (self.workspace.data_ptr() + 255) // 256 * 256
        self.params.workspace_bytes = need.value
        self.frame = 0
        self.prev_cam = None
        # render_graph: captured frames, by (output image, is_active word)
        self._graphs = {}

    def set_time(self, time, is_afternoon):
        """Status.time / Status.is_afternoon of the next frames (sky colour,
        mat.glsl:137-202)."""
        self.status_host[0]["time"] = time
        self.status_host[0]["is_afternoon"] = int(bool(is_afternoon))

    # -- per-frame host->device state -------------------------------------
    def _frame_state(self, inv_view, inv_proj):
        """Fills the host copies of camera_view and Status for the next
        frame; returns its is_active word."""
        c = self.camera_host[0]
        c["inv_view"], c["inv_proj"] = inv_view, inv_proj
        pv, pp = self.prev_cam if self.prev_cam is not None else (inv_view, inv_proj)
        c["prev_inv_view"], c["prev_inv_proj"] = pv, pp
        taa_on = self.taa and self.frame > 0
        s = self.status_host[0]
        s["frame_number"] = self.frame
        remap = L.REMAP_BIT if self.sb.accel_prev is not None else 0
        s["is_active"] = self.features | (L.TAA_BIT if taa_on else 0) | remap
        return int(s["is_active"])

    def _upload(self, inv_view, inv_proj):
        self._frame_state(inv_view, inv_proj)
        s = self.status_host[0]
        slot = self._ring_pos
        self._ring_pos = (slot + 1) % len(self._ring)
        buf, ev = self._ring[slot]
        if self._ring_used[slot]:
            ev.synchronize()
        nc = L.CAMERA_VIEW.itemsize
        host = buf.numpy()
        host[:nc] = self.camera_host.view(np.uint8)
        host[nc:] = self.status_host.view(np.uint8)
        self.camera.copy_(buf[:nc], non_blocking=True)
        self.status.copy_(buf[nc:], non_blocking=True)
        ev.record()
        self._ring_used[slot] = True
        return int(s["is_active"])

    H2D_BYTES_PER_FRAME = 264 + 96  # camera_view + Status

    def push_constant(self):
        cur, prev = self.images[self.frame % 2], self.images[(self.frame + 1) % 2]
        pc = native.PushConstant()
        pc.size[0], pc.size[1] = self.W, self.H
        pc.tlas = self.sb.accel.handle
        pc.tlas_previous = (self.sb.accel_prev or self.sb.accel).handle
        pc.swapchain = cur.data_ptr()
        pc.previous_swapchain = (prev if self.frame > 0 else cur).data_ptr()
        pc.taa_frame = self.taa_frame.data_ptr()
        pc.taa_prev_frame = self.taa_prev.data_ptr()
        pc.camera_buffer = self.camera.data_ptr()
        pc.status_buffer = self.status.data_ptr()
        pc.world_buffer = self.sb.world.data_ptr()
        pc.restir_buffer = self.restir.data_ptr()
        return pc

    # -- frame history checkpoint (ct_state_save / ct_state_load) ----------
    def state_size(self):
        n = ctypes.c_uint64()
        native.check("ct_state_size", native.lib().ct_state_size(self.W, self.H, ctypes.byref(n)))
        return n.value

    def save_state(self):
        """The history the last frame leaves for the next (ct_state_save) as
        a host uint8 array, with the host side's frame number and previous
        camera."""
        blob = torch.empty(self.state_size(), dtype=torch.uint8).pin_memory()
        self.frame -= 1  # the push constant of the frame just rendered
        try:
            pc = self.push_constant()
        finally:
            self.frame += 1
        stream = torch.cuda.current_stream().cuda_stream
        native.check("ct_state_save", native.lib().ct_state_save(ctypes.byref(pc), blob.data_ptr(), blob.numel(),
                                                                 stream))
        return blob.numpy().copy(), self.frame, self.prev_cam

    def load_state(self, state):
        """Continues from a save_state() result: the next render() is the
        frame after the saved one."""
        blob, frame, prev_cam = state
        blob = np.ascontiguousarray(blob, np.uint8)
        self.frame = frame - 1
        try:
            pc = self.push_constant()
        finally:
            self.frame = frame
        self.prev_cam = prev_cam
        stream = torch.cuda.current_stream().cuda_stream
        native.check("ct_state_load", native.lib().ct_state_load(ctypes.byref(pc), blob.ctypes.data, blob.size,
                                                                 stream))

    def _frame_done(self, inv_view, inv_proj):
        """Host bookkeeping after a frame is recorded."""
        self.prev_cam = (np.array(inv_view), np.array(inv_proj))
        self.frame += 1

    def render(self, inv_view, inv_proj, stages=None):
        """Records one frame on the current stream; returns the output image
        tensor (H, W, 4).  `stages` restricts the passes ("trace", "di0",
        "pt0", "di1", "pt1", "taa") for tests."""
        is_active = self._upload(inv_view, inv_proj)
        pc = self.push_constant()
        stream = torch.cuda.current_stream().cuda_stream
        L_ = native.lib()
        p = ctypes.byref(self.params)
        if stages is None:
            native.check("ct_render_frame", L_.ct_render_frame(ctypes.byref(pc), p, is_active, stream))
        else:
            if "trace" in stages:
                native.check("ct_trace_frame", L_.ct_trace_frame(ctypes.byref(pc), p, stream))
            if "di0" in stages:
                native.check("ct_restir_di", L_.ct_restir_di(ctypes.byref(pc), p, 0, stream))
            if "pt0" in stages:
                native.check("ct_restir_pt", L_.ct_restir_pt(ctypes.byref(pc), p, 0, stream))
            if "di1" in stages:
                native.check("ct_restir_di", L_.ct_restir_di(ctypes.byref(pc), p, 1, stream))
            if "pt1" in stages:
                native.check("ct_restir_pt", L_.ct_restir_pt(ctypes.byref(pc), p, 1, stream))
            if "taa" in stages and (is_active & L.TAA_BIT):
                native.check("ct_taa", L_.ct_taa(ctypes.byref(pc), p, stream))
        out = self.images[self.frame % 2]
        self.prev_cam = (np.array(inv_view), np.array(inv_proj))
        self.frame += 1
        if self.sb.accel_prev is not None:
            # settling after an edit: remap tables back to zero for the next
            # edit (clear_instance_remapping_buffer, accel_struct_mngr.cpp:2616-2625)
            self.sb.remap_p.zero_()
            self.sb.remap_l.zero_()
            # freed at the next edit: cudaFree would wait for this frame here
            self.sb.accel_retired.append(self.sb.accel_prev)
            self.sb.accel_prev = None
        return out

    def render_graph(self, inv_view, inv_proj):
        """render(), with the frame's launches replayed from a CUDA graph:
        one launch of the host instead of one per kernel.  The camera and
        Status upload stays outside the graph.  A graph is captured on first
        use for each output image (the two alternate) and status word; the
        first frame and a frame right after an edit run through render()
        (the first sizes the scratch, the second binds the previous scene),
        and an edit's rebuild drops the graphs."""
        if self.frame == 0 or self.sb.accel_prev is not None:
            return self.render(inv_view, inv_proj)
        is_active = self._upload(inv_view, inv_proj)
        key = (self.frame % 2, is_active, self.sb.accel.handle)
        g = self._graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            pc = self.push_constant()
            with torch.cuda.graph(g):
                native.check("ct_render_frame",
                             native.lib().ct_render_frame(ctypes.byref(pc), ctypes.byref(self.params), is_active,
                                                          torch.cuda.current_stream().cuda_stream))
            self._graphs[key] = g
        g.replay()
        out = self.images[self.frame % 2]
        self.prev_cam = (np.array(inv_view), np.array(inv_proj))
        self.frame += 1
        return out

    def erase(self, pixel, window=50):
        """Removes the voxels under a square brush of half width `window`
        pixels around `pixel` of the last rendered frame (ct_brush), keeps
        the primitive ranges dense (ct_rearrange) and rebuilds the
        acceleration structure.  The next frame renders with REMAP_BIT and
        the structure before the edit as tlas_previous.  The default window
        is the reference brush's (brush_mngr.hpp:125)."""
        self.brush(pixel, window)
        self.rearrange()
        self.rebuild()

    def brush(self, pixel, window=50):
        """ct_brush: marks the primitives under the brush in the scene's
        bitmasks (Status.pixel, BRUSH_CONFIG.brush_pixel_size)."""
        s = self.status_host[0]
        s["pixel"] = pixel
        cfg = np.zeros(1, L.BRUSH_CONFIG)
        cfg["brush_type"] = 0
        cfg["brush_pixel_size"] = (window, 0, 0)
        self.sb.brush_config.copy_(torch.from_numpy(cfg.view(np.uint8).copy()).to(self.device))
        self._upload_status()
        pc = self.push_constant_edit()
        native.check("ct_brush", native.lib().ct_brush(ctypes.byref(pc), torch.cuda.current_stream().cuda_stream))

    def rearrange(self):
        """ct_rearrange: removes the marked primitives and their cube lights."""
        pc = self.push_constant_edit()
        native.check("ct_rearrange", native.lib().ct_rearrange(ctypes.byref(pc), self.sb.n_instances,
                                                               self.sb.n_primitives,
                                                               torch.cuda.current_stream().cuda_stream))

    def rebuild(self):
        """New acceleration structure over the edited buffers; the old one
        stays bound as tlas_previous for the next frame."""
        for a in self.sb.accel_retired:
            a.free()
        self.sb.accel_retired.clear()
        if self.sb.accel_prev is not None:
            self.sb.accel_prev.free()
        self._graphs.clear()
        self.sb.accel_prev = self.sb.accel
        self.sb.accel = Accel(self.sb.instances, self.sb.n_instances, self.sb.aabbs, self.sb.n_primitives,
                              self.scene.voxel_extent)

    def scene_state(self):
        """Host copies of the scene tables an edit changes."""
        torch.cuda.synchronize()
        sb = self.sb
        n_cube = max(self.scene.cube_lights.shape[0], 1)

        def arr(t, dt, n=None):
            a = t.cpu().numpy().view(np.uint8).view(dt)
            return a if n is None else a[:n]
        return {
            "instances": arr(sb.instances, L.INSTANCE, sb.n_instances),
            "primitives": arr(sb.primitives, L.PRIMITIVE, sb.n_primitives),
            "aabbs": arr(sb.aabbs, L.AABB, sb.n_primitives),
            "cube_lights": arr(sb.cube_lights, L.LIGHT, n_cube),
            "light_config": arr(sb.light_config, L.LIGHT_CONFIG, 1),
            "remap_p": sb.remap_p.cpu().numpy().view(np.uint32)[:sb.n_primitives],
            "remap_l": sb.remap_l.cpu().numpy().view(np.uint32)[:n_cube],
            "primitive_bitmask": sb.primitive_bitmask.cpu().numpy().view(np.uint32),
            "instance_bitmask": sb.instance_bitmask.cpu().numpy().view(np.uint32),
            "brush_counter": sb.brush_counter.cpu().numpy().view(np.uint32),
        }

    def _upload_status(self):
        host = torch.from_numpy(self.status_host.view(np.uint8).copy())
        self.status.copy_(host.to(self.device))

    def push_constant_edit(self):
        """The push constant of the edit passes (the last frame's buffers)."""
        pc = native.PushConstant()
        pc.size[0], pc.size[1] = self.W, self.H
        pc.tlas = pc.tlas_previous = self.sb.accel.handle
        pc.camera_buffer = self.camera.data_ptr()
        pc.status_buffer = self.status.data_ptr()
        pc.world_buffer = self.sb.world.data_ptr()
        pc.restir_buffer = self.restir.data_ptr()
        return pc

    def device_error(self, reset=True):
        e = native.ErrorInfo()
        native.check("ct_get_error", native.lib().ct_get_error(torch.cuda.current_stream().cuda_stream, int(reset),
                                                               ctypes.byref(e)))
        return e.status, e.detail, e.pixel

    def read(self, key):
        """Host copy of a per-pixel buffer as a structured array."""
        return L.view_buffer(key, self.buf[key].cpu().numpy())

    COUNTER_NAMES = ("primary", "shadow", "bounce", "voxel_tests", "brick_visits", "candidates", "neighbours",
                     "temporal", "hits", "bounce_hits", "walker_bricks")

    def ray_counts(self, reset=True):
        """Work counters accumulated since the last reset (needs count_rays=True)."""
        c = self.counters.cpu().numpy()
        if reset:
            self.counters.zero_()
        return {n: int(c[i]) for i, n in enumerate(self.COUNTER_NAMES)}
