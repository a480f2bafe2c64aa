"""Many views rendered side by side: one ct_render_views call per frame,
replayed from a captured CUDA graph, with a schedule picked by measurement.

The reference renders one view per frame (App::draw, src/main.cpp:1436-1703);
this batches independent views, each with its own per-pixel buffers and
scratch, over scenes that views may share.  Per view the frame is exactly
the one Renderer.render records (the same entry points in App::draw's
order), so a view rendered in a batch matches the same view rendered alone
bit for bit.

  views_workload      -- seeded scenes of the 64^3 kind with edges
                         log-uniform in [64, 512], occupancy U[0.1, 0.4],
                         and views of log-uniform resolution on them
  MultiViewRenderer   -- the batch: one packed camera/Status upload, one
                         ct_render_views (a graph replay after the first
                         frame) per frame
  MultiViewRenderer.autotune -- times candidate schedules (lane count,
                         walker grid per view) and keeps the fastest

A schedule assigns views to lanes (streams that become concurrent graph
branches) by longest-processing-time order on the views' pixel counts, and
sets each view's persistent-walker grid (ct_params.walker_blocks): the
library default (8 blocks per SM) or a grid proportional to the view's
pixel count.
"""
import ctypes
import math

import numpy as np
import torch

from . import layouts as L
from . import native
from . import scenes
from .frame import Renderer, SceneBuffers

BLOCK = L.CAMERA_VIEW.itemsize + L.STATUS.itemsize  # 360 B of per-frame upload per view


def views_workload(n_scenes=8, n_views=32, seed=2024, edge_range=(64, 512), occupancy_range=(0.1, 0.4),
                   res_min=(128, 128), res_max=(1920, 1080), step=0.1):
    """(scenes, views): n_scenes random grids (config-0 kind: 2% emitters with
    radiance U[1,10], albedo U[0.2,0.8]) with edge log-uniform in
    edge_range and occupancy uniform in occupancy_range; n_views views,
    view i on scene i % n_scenes, width and height log-uniform between
    res_min and res_max, the eye outside the grid at a seeded direction
    looking at its centre, moving `step` * edge / 64 along x per frame.
    Each view is a dict (scene index, width, height, eye, target, step)."""
    rng = np.random.default_rng(seed)
    out_scenes = []
    for k in range(n_scenes):
        edge = int(round(math.exp(rng.uniform(math.log(edge_range[0]), math.log(edge_range[1])))))
        occ = float(rng.uniform(*occupancy_range))
        sc = scenes.random_grid_scene(edge, occ, emissive_fraction=0.02, seed=int(rng.integers(1 << 30)),
                                      albedo=(0.2, 0.8), radiance=(1.0, 10.0))
        out_scenes.append(sc)
    views = []
    for i in range(n_views):
        k = i % n_scenes
        edge = out_scenes[k].grid_edge[0]
        w = int(round(math.exp(rng.uniform(math.log(res_min[0]), math.log(res_max[0])))))
        h = int(round(math.exp(rng.uniform(math.log(res_min[1]), math.log(res_max[1])))))
        az = rng.uniform(0.0, 2.0 * math.pi)
        el = rng.uniform(0.3, 0.9)
        c = np.array([edge * 0.5] * 3)
        r = edge * 1.2
        eye = c + r * np.array([math.cos(az) * math.cos(el), math.sin(el), math.sin(az) * math.cos(el)])
        views.append({"scene": k, "width": w, "height": h, "eye": eye, "target": c,
                      "step": np.array([step * edge / 64.0, 0.0, 0.0])})
    return out_scenes, views


def view_cameras(view, frame):
    return scenes.camera_matrices(view["eye"] + frame * view["step"], view["target"] + frame * view["step"],
                                  view["width"], view["height"], 60.0)


class MultiViewRenderer:
    """Renderers of many views, recorded together by ct_render_views."""

    def __init__(self, scene_list, views, device="cuda", **renderer_kw):
        self.device = device
        self.sbs = [SceneBuffers(sc, device) for sc in scene_list]
        self.views = views
        self.r = [Renderer(self.sbs[v["scene"]].scene, v["width"], v["height"], scene_buffers=self.sbs[v["scene"]],
                           device=device, **renderer_kw) for v in views]
        n = len(self.r)
        # every view's camera_view and Status in one device buffer, uploaded
        # from one pinned buffer per frame
        self.dev_blocks = torch.zeros(n * BLOCK, dtype=torch.uint8, device=device)
        self.host_blocks = [torch.zeros(n * BLOCK, dtype=torch.uint8).pin_memory() for _ in range(2)]
        self.host_ev = [None, None]
        self.host_pos = 0
        nc = L.CAMERA_VIEW.itemsize
        for i, r in enumerate(self.r):
            r.camera = self.dev_blocks[i * BLOCK:i * BLOCK + nc]
            r.status = self.dev_blocks[i * BLOCK + nc:(i + 1) * BLOCK]
        self.lanes = []
        self.frame = 0
        self._graphs = {}
        self.n_sm = torch.cuda.get_device_properties(device).multi_processor_count
        self.set_schedule(lanes=min(8, n), walker="default")

    @property
    def pixels(self):
        return [r.W * r.H for r in self.r]

    def set_schedule(self, lanes, walker="default"):
        """lanes: streams the views are spread over (0: all on the current
        stream, in order); walker: "default" (8 blocks per SM per view) or
        "proportional" (blocks in proportion to the view's pixels, a
        1920x1080 view getting the default)."""
        px = self.pixels
        self.lane_of = [0] * len(px)
        if lanes > 0:
            load = [0] * lanes
            for i in sorted(range(len(px)), key=lambda i: -px[i]):
                lane = int(np.argmin(load))
                self.lane_of[i] = lane
                load[lane] += px[i]
        while len(self.lanes) < lanes:
            self.lanes.append(torch.cuda.Stream(self.device))
        self.n_lanes = lanes
        full = self.n_sm * 8
        for r, p in zip(self.r, px):
            r.params.walker_blocks = 0 if walker == "default" else max(16, min(full, math.ceil(full * p / (1920 * 1080))))
        self.schedule = {"lanes": lanes, "walker": walker}
        self._graphs.clear()

    def _upload(self, cams):
        host = self.host_blocks[self.host_pos]
        ev = self.host_ev[self.host_pos]
        if ev is not None:
            ev.synchronize()
        arr = host.numpy()
        nc = L.CAMERA_VIEW.itemsize
        actives = []
        for i, (r, (iv, ip)) in enumerate(zip(self.r, cams)):
            actives.append(r._frame_state(iv, ip))
            arr[i * BLOCK:i * BLOCK + nc] = r.camera_host.view(np.uint8)
            arr[i * BLOCK + nc:(i + 1) * BLOCK] = r.status_host.view(np.uint8)
        self.dev_blocks.copy_(host, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self.host_ev[self.host_pos] = ev
        self.host_pos ^= 1
        return actives

    def _views(self, actives):
        arr = (native.View * len(self.r))()
        for i, r in enumerate(self.r):
            arr[i].pc = r.push_constant()
            arr[i].params = r.params
            arr[i].is_active = actives[i]
            arr[i].lane = self.lane_of[i]
        return arr

    def _record(self, actives):
        views = self._views(actives)
        lanes = (ctypes.c_void_p * max(self.n_lanes, 1))(*[s.cuda_stream for s in self.lanes[:self.n_lanes]])
        native.check("ct_render_views", native.lib().ct_render_views(
            views, len(self.r), lanes, self.n_lanes, torch.cuda.current_stream().cuda_stream))

    def render(self, cams, graph=True):
        """One frame of every view (cams: (inv_view, inv_proj) per view).
        After the first frame, the frame's launches are replayed from a CUDA
        graph captured once per output-image parity and status words."""
        actives = self._upload(cams)
        if not graph or self.frame == 0:
            self._record(actives)
        else:
            key = (self.frame % 2, tuple(actives))
            g = self._graphs.get(key)
            if g is None:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._record(actives)
                self._graphs[key] = g
            g.replay()
        for r, (iv, ip) in zip(self.r, cams):
            r._frame_done(iv, ip)
        self.frame += 1

    def render_sequential(self, cams):
        """The baseline: every view's ct_render_frame in turn on the current
        stream, no graph."""
        for r, (iv, ip) in zip(self.r, cams):
            r.render(iv, ip)
        self.frame += 1

    def cams(self, frame):
        return [view_cameras(v, frame) for v in self.views]

    def autotune(self, lanes_options=(0, 2, 4, 8, 16, 32), walker_options=("default", "proportional"), frames=3):
        """Times every (lanes, walker) schedule on `frames` graph replays
        after a capture frame and keeps the fastest.  Returns the table of
        (lanes, walker, ms per frame), fastest first."""
        table = []
        for lanes in lanes_options:
            if lanes > len(self.r):
                continue
            for walker in walker_options:
                self.set_schedule(lanes, walker)
                for _ in range(2):  # capture both image parities
                    self.render(self.cams(self.frame))
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(frames):
                    self.render(self.cams(self.frame))
                e1.record()
                torch.cuda.synchronize()
                table.append((lanes, walker, e0.elapsed_time(e1) / frames))
        table.sort(key=lambda t: t[2])
        self.set_schedule(table[0][0], table[0][1])
        self.autotune_table = table
        return table

    def device_error(self):
        return self.r[0].device_error()
