#!/usr/bin/env python3
"""Benchmark of the voxel ray-tracing frame (the terrain workload at 1080p).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: 256^3 heightfield terrain (h = 64 + 48 * 4-octave seeded value
noise, ~4.2M voxel AABBs, 0.5% of the surface voxels are cube lights with
radiance U[2,20], albedo U[0.1,0.9]), 1920x1080, orbit camera; per frame:
primary rays, ReSTIR DI with 32 cube-light candidates, temporal reuse and 2
spatial rounds, ReSTIR PT to depth 8 with the hybrid shift and temporal and
spatial path reuse, TAA with history weight 0.9.  The scene and the per-pixel
state (~0.9 GB) are far larger than the 126 MB L2, so no L2 flush is needed
between frames.  Synthetic seeded data; no dataset is involved.

A step is one frame.  `value` is Mrays/s over all ranks (primary + shadow +
bounce rays actually traced, counted by the kernels in an untimed replay of
the same frames) with all inputs resident on the device; `ms_per_step` is
ms/frame.  `e2e` is the same metric through the C ABI with the per-frame
camera/Status upload from pinned host memory and the read-back of the output
image inside the timed region.

--impl reference times the reference's own shader code compiled for the
host (oracle/_ref, the reference's GLSL built as C++) on all host cores,
on a bounded sample of the same workload (a band of image rows) with the
same run-time parameters, rank 0 only.  The default run also reports
`fp64_error` (untimed): on that band, the error of the CUDA frame against
the double-precision build of the same shader code continuing the CUDA
run's saved history.

Multi-GPU: views are independent, so N ranks render N replicas (no
collective on the data path); `value` = rays of all ranks / max time.
"""
import argparse
import json
import os
import subprocess
import threading
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cube-tracing_b200"))

W_DEFAULT, H_DEFAULT = 1920, 1080
METRIC = "ms/frame & Mrays/s at 1080p"


MAX_DEPTH = 8


def workload(edge=256):
    """256^3 heightfield terrain, 0.5% of surface voxels emissive, plus one
    point light above the terrain (the only light kind ReSTIR PT's next event
    estimation samples, path_tracer.glsl:218-255)."""
    import numpy as np
    from cube_tracing import layouts as L
    from cube_tracing import scenes
    sc = scenes.heightfield_scene(edge, base=64.0, amplitude=48.0, emissive_fraction=0.005, seed=1,
                                  albedo=(0.1, 0.9), radiance=(2.0, 20.0))
    pl = np.zeros(1, L.LIGHT)
    pl["position"] = (edge * 0.5, edge * 1.5, edge * 0.5)
    pl["emissive"] = (4.0, 4.0, 4.0)
    pl["instance_id"] = L.MAX_INSTANCES
    pl["primitive_id"] = L.MAX_PRIMITIVES
    pl["type"] = L.LIGHT_POINT
    sc.point_lights = pl
    sc.light_config["point_light_count"] = 1
    return sc


def headline_params():
    """The workload's reuse parameters, as ct_params overrides (the CUDA
    path) and oracle run-time parameters (the reference's shaders): 32
    cube-light candidates, 2 DI spatial rounds, TAA keeping 0.9 of the
    history (current-frame weight 0.1), and ReSTIR PT's hybrid shift with a
    0.5-unit near-field distance (the reconnection vertex is the first whose
    incoming segment is at least 0.5 units long and which, with its
    predecessor, is diffuse)."""
    return {"max_ris_cube_samples": 32, "spatial_passes": 2, "taa_alpha": 0.1, "pt_shift_mapping": 2,
            "pt_near_field_distance": 0.5}


def camera_frames(n, W, H):
    from cube_tracing import scenes
    return scenes.camera_path("orbit", n, W, H, center=(128.0, 60.0, 128.0), radius=140.0, elevation=90.0,
                              deg_per_frame=0.5)


def config_dict(sc, W, H, extra=None):
    d = {"workload": "terrain256_1080p", "scene": "heightfield 256^3, 4-octave value noise, 0.5% emissive surface",
         "voxels": sc.voxel_count, "cube_lights": int(sc.cube_lights.shape[0]), "resolution": [W, H],
         "spp": 1, "ris_cube_candidates": 32, "temporal": True, "spatial_rounds": 2, "spatial_neighbours": "3-4",
         "spatial_radius_px": "2-50", "taa_history_weight": 0.9,
         "point_lights": int(sc.point_lights.shape[0]),
         "pt": f"ReSTIR PT, hybrid shift (reconnect at the first vertex whose incoming segment is >= 0.5 units "
               f"and which, with its predecessor, is diffuse; random replay before it), max depth {MAX_DEPTH}, "
               f"temporal + spatial path reuse",
         "camera": "orbit r=140 elev=90 around (128,60,128), 0.5 deg/frame", "l2_flush": "not needed: scene + per-pixel state > 126 MB L2"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(gpu_index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def wait_ready(self, timeout=10.0):
        """Blocks until nvidia-smi printed its first sample: its start-up
        (driver queries, a few hundred ms of host time) then lies before the
        timed region instead of inside it."""
        self.first = ""
        if self.proc is None:
            return self
        ready = threading.Event()

        def first_line():
            self.first = self.proc.stdout.readline()
            ready.set()

        threading.Thread(target=first_line, daemon=True).start()
        ready.wait(timeout)
        return self

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        out = getattr(self, "first", "") + out
        rows = [r.split(",") for r in out.strip().splitlines() if r.strip()]
        sm = [float(r[0]) for r in rows if len(r) >= 8 and r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if len(r) >= 8 and r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 8:
                continue
            for i, n in enumerate(names):
                if r[4 + i].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(rows), "reasons": sorted(reasons)}


def measured_peaks(key="hbm_gbs"):
    """A peak from MEASURED_PEAKS.json (hbm_gbs, bf16_tflops, ...), else the
    earlier measurement on these GPUs."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if key in d:
            return float(d[key]), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}[key], "fallback"


def profile_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None, None
    with open(p) as f:
        d = json.load(f)
    e = d.get(kernel)
    if not e:
        return None, None
    return e.get("bytes_per_launch_full_frame"), e.get("note")


def combine_ranks(ms_per_step, e2e_ms_per_step, rays, world, device, wall_ms_per_step=None):
    """Whole-job figures of N independent replicas: the slowest rank's device
    times and the rays of all ranks (torch.distributed, any backend).  With
    `wall_ms_per_step` (a host clock) its maximum over ranks is returned as a
    fourth value."""
    if world <= 1:
        out = (ms_per_step, e2e_ms_per_step, float(rays))
        return out if wall_ms_per_step is None else out + (wall_ms_per_step,)
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms_per_step, e2e_ms_per_step, wall_ms_per_step or 0.0], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    r = torch.tensor([float(rays)], device=device, dtype=torch.float64)
    dist.all_reduce(r)
    out = (float(t[0]), float(t[1]), float(r[0]))
    return out if wall_ms_per_step is None else out + (float(t[2]),)


# ---------------------------------------------------------------------------
def run_b200(args, rank, world):
    import ctypes

    import torch
    from cube_tracing import accounting as acct
    from cube_tracing import layouts as L
    from cube_tracing import native
    from cube_tracing.frame import Renderer, SceneBuffers

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    W, H = args.width, args.height
    sc = workload(args.edge)
    sb = SceneBuffers(sc, device=dev)
    n_frames = args.warmup + args.steps
    cams = camera_frames(n_frames + 8, W, H)
    lib = native.lib()

    def make_renderer(**kw):
        params = native.params_for_scene(sc, **headline_params())
        return Renderer(sc, W, H, params=params, scene_buffers=sb, device=dev, indirect=True, max_depth=MAX_DEPTH,
                        **kw)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # the frame's entry points in App::draw order
    STAGES = [("k_trace_primary", "ct_trace_frame", None), ("k_di_initial", "ct_restir_di", 0),
              ("k_pt_trace", "ct_restir_pt", 0), ("k_di_shade", "ct_restir_di", 1),
              ("k_pt_spatial", "ct_restir_pt", 1), ("k_taa", "ct_taa", None)]

    def run_stages(rr, cam, after_stage=None):
        is_active = rr._upload(*cam)
        pc = rr.push_constant()
        p = ctypes.byref(rr.params)
        s = torch.cuda.current_stream().cuda_stream
        for name, fn, stage in STAGES:
            if fn == "ct_taa" and not (is_active & L.TAA_BIT):
                continue
            args_ = (ctypes.byref(pc), p) + ((stage,) if stage is not None else ()) + (s,)
            native.check(fn, getattr(lib, fn)(*args_))
            if after_stage:
                after_stage(name)
        rr.prev_cam = (np.array(cam[0]), np.array(cam[1]))
        rr.frame += 1
        return is_active

    # --- device-resident timing -------------------------------------------
    r = make_renderer()
    clocks = ClockSampler(dev.index if dev.index is not None else 0).wait_ready()
    for f in range(args.warmup):
        r.render(*cams[f])
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        r.render(*cams[args.warmup + k])
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    err = r.device_error()
    if err[0] != 0:
        raise RuntimeError(f"device error {err}")

    # --- per-stage timing (CUDA events between entry points) and per-kernel
    # timing (events around every launch, ct_profile_enable) on the same
    # renderer, continuing the orbit ----------------------------------------
    stage_ms = {name: 0.0 for name, _, _ in STAGES}
    n_stage_frames = 4
    for f in range(n_stage_frames):
        marks = []

        def mark(name):
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            marks.append((name, ev))

        start = torch.cuda.Event(enable_timing=True)
        start.record()
        run_stages(r, cams[n_frames + f], mark)
        torch.cuda.synchronize()
        prev = start
        for name, ev in marks:
            stage_ms[name] += prev.elapsed_time(ev) / n_stage_frames
            prev = ev
    native.check("ct_profile_enable", lib.ct_profile_enable(1))
    native.kernel_times(reset=True)
    for f in range(n_stage_frames):
        r.render(*cams[n_frames + n_stage_frames + f])
    torch.cuda.synchronize()
    ktimes = native.kernel_times(reset=True)
    native.check("ct_profile_enable", lib.ct_profile_enable(0))
    kernel_ms = {k: (ms / n_stage_frames, n // n_stage_frames) for k, (ms, n) in ktimes.items()}
    launches_per_frame = sum(n for _, n in kernel_ms.values())
    del r

    # --- e2e through the C ABI with host buffers ---------------------------
    # Each frame's image goes back to pinned host memory on a copy stream
    # while the next frame renders: a frame writes one of the renderer's two
    # output images and only reads the other (TAA history), so frame k + 2,
    # which writes frame k's image again, waits for that image's copy.
    host_img = [torch.empty((H, W, 4), dtype=torch.float32).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream(dev)
    r2 = make_renderer()
    for f in range(args.warmup):
        r2.render(*cams[f])
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    copied = [None, None]
    main = torch.cuda.current_stream(dev)
    wall0 = time.perf_counter()
    t0.record()
    for k in range(args.steps):
        if copied[k % 2] is not None:
            main.wait_event(copied[k % 2])
        img = r2.render(*cams[args.warmup + k])
        rendered = torch.cuda.Event()
        rendered.record(main)
        copy_stream.wait_event(rendered)
        with torch.cuda.stream(copy_stream):
            host_img[k % 2].copy_(img, non_blocking=True)
        copied[k % 2] = torch.cuda.Event()
        copied[k % 2].record(copy_stream)
    for ev in copied:
        if ev is not None:
            main.wait_event(ev)
    t1.record()
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - wall0) * 1e3
    barrier()
    e2e_ms = t0.elapsed_time(t1)
    del r2

    # --- untimed replay with work counters ---------------------------------
    rc = make_renderer(count_rays=True)
    for f in range(args.warmup):
        rc.render(*cams[f])
    torch.cuda.synchronize()
    rc.ray_counts(reset=True)
    for k in range(args.steps):
        rc.render(*cams[args.warmup + k])
    torch.cuda.synchronize()
    totals = rc.ray_counts(reset=True)
    # one more frame stage by stage for the per-kernel byte counts
    per_stage = {}

    def grab(name):
        torch.cuda.synchronize()
        per_stage[name] = rc.ray_counts(reset=True)

    is_active = run_stages(rc, cams[n_frames], grab)
    pixels = W * H
    hits = per_stage["k_trace_primary"]["hits"]
    taa = bool(is_active & L.TAA_BIT)
    spatial = rc.params.spatial_passes
    c1 = per_stage["k_di_shade"]
    hits_frame = c1["hits"] // spatial
    di1 = (c1["hits"] * (acct.DI + acct.RES + acct.MAT) + hits_frame * ((spatial - 1) * acct.RES + acct.RES + acct.DI) +
           (pixels - hits_frame) * 4 + c1["neighbours"] * (acct.DI + acct.RES + acct.MAT) +
           c1["brick_visits"] * acct.BRICK)
    taa_pixels = (W // 8) * (H // 8) * 64
    b_alg = {
        "k_trace_primary": acct.trace_bytes(per_stage["k_trace_primary"], pixels, taa),
        "k_di_initial": acct.di_initial_bytes(per_stage["k_di_initial"]),
        "k_pt_trace": acct.pt_trace_bytes(per_stage["k_pt_trace"]),
        "k_di_shade": di1,
        "k_pt_spatial": acct.pt_spatial_bytes(per_stage["k_pt_spatial"], taa),
        "k_taa": acct.taa_bytes(int(hits * taa_pixels / pixels), taa_pixels) if taa else 0,
    }

    rays = totals["primary"] + totals["shadow"] + totals["bounce"]
    ms_per_step, e2e_ms_step, rays_all, wall_ms_step = combine_ranks(ms_total / args.steps, e2e_ms / args.steps, rays,
                                                                     world, dev, wall_ms / args.steps)
    mrays = rays_all / (ms_per_step * args.steps / 1e3) / 1e6
    mrays_e2e = rays_all / (e2e_ms_step * args.steps / 1e3) / 1e6

    # Roofline of the dominant kernel.  Algorithmic bytes per launch: for the
    # shadow-ray walker, the 64 B occupancy mask of every 8^3 brick its rays
    # enter (its own brick counter over the frame / its launches); for the
    # single-launch stage kernels (primary trace, PT spatial, TAA) the
    # stage's bytes.
    dom = max(kernel_ms, key=lambda k: kernel_ms[k][0])
    peak, peak_kind = measured_peaks()
    dom_ms, dom_launches = kernel_ms[dom]
    t_launch = dom_ms / max(dom_launches, 1) / 1e3
    if dom == "k_trace_shadow":
        shadow_bricks = sum(c["walker_bricks"] for c in per_stage.values())
        bytes_launch = shadow_bricks * acct.BRICK / max(dom_launches, 1)
    else:
        bytes_launch = b_alg.get(dom, 0)
    achieved = bytes_launch / t_launch / 1e9 if t_launch > 0 else 0.0
    traffic, traffic_note = profile_traffic(dom)
    result = {
        "metric": METRIC, "value": round(mrays, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded heightfield terrain, orbit camera)",
        "config": config_dict(sc, W, H, {"parallelism": f"replicas x{world}" if world > 1 else "single view"}),
        "rays_per_frame": {k: totals[k] // args.steps for k in ("primary", "shadow", "bounce")},
        "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "kernel_ms_per_frame": {k: round(v[0], 4) for k, v in sorted(kernel_ms.items(), key=lambda kv: -kv[1][0])},
        "e2e": {"value": round(mrays_e2e, 2), "unit": "Mrays/s", "ms_per_step": round(e2e_ms_step, 4),
                "h2d_bytes_per_step": Renderer.H2D_BYTES_PER_FRAME, "d2h_bytes_per_step": W * H * 16,
                "host_wall_ms_per_step": round(wall_ms_step, 4),
                "host_wall_value": round(rays_all / (wall_ms_step * args.steps / 1e3) / 1e6, 2)
                if wall_ms_step > 0 else None,
                "timing": "value/ms_per_step: CUDA events on the rendering stream, the last frame's image "
                          "copy waited for; each image is copied back on a copy stream while the next frame "
                          "renders; host_wall_*: time.perf_counter around the same loop, ending after a "
                          "device synchronize"},
        "gpu_launches": launches_per_frame * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "launches_per_frame": dom_launches,
                     "ms_per_launch": round(t_launch * 1e3, 4),
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": int(bytes_launch),
                     "traffic": traffic, "traffic_note": traffic_note},
        "clocks": clk,
    }
    return result


# ---------------------------------------------------------------------------
# rows of the frame the last row of a band depends on, beyond the band: two DI
# spatial rounds of at most 50 px each, TAA's 3x3 window, PT's 1-px spatial
# reuse (the previous frame's buffers come whole from the saved history)
BAND_MARGIN = 128


def band_rows(H, rows):
    rows = max(1, min(H, rows))
    r0 = (H - rows) // 2
    return r0, r0 + rows


def cuda_fp64_error(gpu, sc, W, H, cams, band, threads=0):
    """Error of a CUDA frame against the FP64 build of the oracle (the
    reference's shaders in double precision) on the same inputs: the CUDA
    renderer `gpu` renders cams[:-1], saves its history (ct_state_save) and
    renders the last frame; the FP64 oracle loads that history and renders
    the last frame over `band` with BAND_MARGIN rows on either side, so that
    every pixel of the band sees the inputs it sees in the full frame.
    Returns pyoracle.precision_error over the band (choices that agree, and
    the image's relative error)."""
    import types

    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    for cam in cams[:-1]:
        gpu.render(*cam)
    state = gpu.save_state()
    img = gpu.render(*cams[-1])
    torch.cuda.synchronize()
    keys = ["di", "previous_reservoir", "output_path_reservoir"]
    cuda = types.SimpleNamespace(W=W, H=H, indirect=True, buf={k: gpu.read(k) for k in keys})
    img = img.cpu().numpy()
    r64 = pyoracle.OracleRenderer(sc, W, H, threads=threads, indirect=True, max_depth=MAX_DEPTH, fp64=True,
                                  params=headline_params())
    r64.load_state(state)
    rows = (max(0, band[0] - BAND_MARGIN), min(H, band[1] + BAND_MARGIN))
    img64 = r64.render(*cams[-1], rows=rows)
    err = pyoracle.precision_error(cuda, r64, img, img64, rows=band)
    r64.close()
    err["sample"] = (f"rows {band[0]}-{band[1]} of frame {len(cams) - 1}: the CUDA frame against the FP64 build of "
                     f"the reference's shaders continuing the CUDA run's saved history (rendered over rows "
                     f"{rows[0]}-{rows[1]})")
    return err


def oracle_sample(args):
    """The reference's shaders (oracle/_ref) on host cores over a band of
    rows of the same workload, with the same run-time parameters."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if not pyoracle.available():
        return None, "oracle/_ref/libct_oracle.so not built"
    W, H = args.width, args.height
    sc = workload(args.edge)
    cams = camera_frames(3, W, H)
    threads = os.cpu_count() or 1
    r = pyoracle.OracleRenderer(sc, W, H, threads=threads, indirect=True, max_depth=MAX_DEPTH,
                                params=headline_params())
    band = band_rows(H, args.ref_rows)
    r.render(*cams[0], rows=band)  # fills the band's history
    pyoracle.OracleRenderer.counters(reset=True)
    t = time.perf_counter()
    r.render(*cams[1], rows=band)
    dt = time.perf_counter() - t
    c = pyoracle.OracleRenderer.counters(reset=True)
    rays = c["primary"] + c["shadow"] + c["bounce"]
    r.close()
    mrays = rays / dt / 1e6
    ms_frame = dt * 1e3 * H / (band[1] - band[0])
    sample = (f"rows {band[0]}-{band[1]} of a {W}x{H} frame (frame 2 of the orbit after one warm frame on the same "
              f"band), all three passes of the reference's shaders with INDIRECT_ILLUMINATION_ON (ReSTIR PT, depth "
              f"{MAX_DEPTH}) and the workload's run-time parameters (2 DI spatial rounds, TAA alpha 0.1, hybrid "
              f"shift); "
              f"{rays} rays in {dt:.2f} s; ms/frame extrapolated by rows")
    return {"value": round(mrays, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "ms_per_frame": round(ms_frame, 1), "sample": sample, "voxels": sc.voxel_count}, None


def fp64_error_line(args):
    """cuda_fp64_error on the headline workload (untimed): frame 2 of the
    orbit, the CPU baseline's band of rows."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if not pyoracle.available(fp64=True):
        return {"unavailable": "oracle/_ref/libct_oracle64.so not built"}
    import torch
    from cube_tracing.frame import Renderer
    W, H = args.width, args.height
    sc = workload(args.edge)
    gpu = Renderer(sc, W, H, params=headline_params(), indirect=True, max_depth=MAX_DEPTH,
                   device=torch.device("cuda", torch.cuda.current_device()))
    err = cuda_fp64_error(gpu, sc, W, H, camera_frames(3, W, H), band_rows(H, args.ref_rows),
                          threads=os.cpu_count() or 1)
    del gpu
    return err


def run_reference(args, rank, world):
    if rank != 0:
        return None
    base, why = oracle_sample(args)
    if base is None:
        return {"impl": "reference", "unavailable": why}
    W, H = args.width, args.height
    sc = workload(args.edge)
    return {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": base["ms_per_frame"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded heightfield terrain, orbit camera)",
        "config": config_dict(sc, W, H, {"parallelism": "host threads"}),
        "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": base["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
def run_views(args, rank, world):
    """The many-view workload: 32 views over 8 seeded random grids (edges
    log-uniform in [64, 512], occupancy U[0.1, 0.4]), resolutions
    log-uniform between 128x128 and 1920x1080, DI with one temporal and one
    spatial pass, ReSTIR PT to depth 6, TAA.  A step renders every view
    once.  Timed two ways on the same views, frames continuing: the batch
    (one ct_render_views per frame, replayed from a CUDA graph, with the
    schedule the autotuner picked) and the baseline of 32 ct_render_frame
    calls one after another.  With N ranks each renders the whole set
    (replicas)."""
    import torch
    from cube_tracing import views
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    scs, vs = views.views_workload()
    kw = {"indirect": True, "max_depth": 6}
    mv = views.MultiViewRenderer(scs, vs, device=dev, **kw)
    for _ in range(2):
        mv.render(mv.cams(mv.frame), graph=False)
    table = mv.autotune()
    f0 = mv.frame
    clocks = ClockSampler(dev.index if dev.index is not None else 0).wait_ready()
    for k in range(args.warmup):
        mv.render(mv.cams(f0 + k))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(args.steps):
        mv.render(mv.cams(f0 + args.warmup + k))
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    batch_ms = e0.elapsed_time(e1) / args.steps
    err = mv.device_error()
    if err[0] != 0:
        raise RuntimeError(f"device error {err}")
    # the baseline on the same views, continuing the frames
    f1 = mv.frame
    for k in range(args.warmup):
        mv.render_sequential(mv.cams(f1 + k))
    torch.cuda.synchronize()
    e0.record()
    for k in range(args.steps):
        mv.render_sequential(mv.cams(f1 + args.warmup + k))
    e1.record()
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1) / args.steps
    # rays of one frame of every view, counted in an untimed replay
    rays = 0
    for r in mv.r:
        r.params.flags |= native_flag_count_rays()
        r.params.counters_address = r.counters.data_ptr()
    mv.render_sequential(mv.cams(mv.frame))
    torch.cuda.synchronize()
    for r in mv.r:
        c = r.ray_counts(reset=True)
        rays += c["primary"] + c["shadow"] + c["bounce"]
    px = mv.pixels
    return {
        "metric": "ms/frame of 32 views (batched, one graph launch) and Mrays/s", "value": round(rays / batch_ms / 1e3, 2),
        "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(batch_ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded random grids, seeded views)",
        "config": {"workload": "views32", "scenes": [[int(sc.grid_edge[0]), sc.voxel_count] for sc in scs],
                   "views": [[r.W, r.H] for r in mv.r], "pixels": int(sum(px)), "spp": 1, "max_depth": 6,
                   "di": "32 cube candidates, 1 temporal + 1 spatial pass", "pt": "ReSTIR PT, reconnection shift",
                   "l2_flush": "not needed: scenes + per-pixel state > 126 MB L2"},
        "sequential_ms_per_step": round(seq_ms, 4), "speedup_vs_sequential": round(seq_ms / batch_ms, 3),
        "rays_per_step": int(rays), "schedule": mv.schedule,
        "autotune": [[t[0], t[1], round(t[2], 4)] for t in table], "clocks": clk,
    }


def run_nrc(args, rank, world):
    """The neural radiance cache against the plain tracer.  Scene: the
    terrain scaled to 512^3 (h = 128 + 96 noise, 0.5% emissive surface
    voxels, albedo U[0.1, 0.9]) with a grey sky (miss radiance 0.5), 1920x1080,
    the orbit camera scaled with it.  Plain: the path tracer of
    ct_adjoint_forward at depth 8.  Cache: the same tracer stopped at path
    vertex 2 (the camera is vertex 0: the first bounce hit; ct_nrc_trace with
    cache_vertex 1) with the fused tcgen05 MLP's prediction there, trained
    online on 2^16 self-training paths extended 4 bounces per frame (Adam, lr
    1e-3).  Reference: the plain tracer at 4096 spp.  relMSE = mean of
    (I - R)^2 / (R^2 + 0.01) over pixels and channels.  A step is one cache
    frame (trace + train + infer + compose)."""
    import math
    import torch
    from cube_tracing import adjoint, nrc, scenes
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    edge = 512
    W, H = args.width, args.height
    sc = scenes.heightfield_scene(edge, base=128.0, amplitude=96.0, emissive_fraction=0.005, seed=1,
                                  albedo=(0.1, 0.9), radiance=(2.0, 20.0))
    iv, ip = scenes.camera_path("orbit", 1, W, H, center=(256.0, 120.0, 256.0), radius=280.0, elevation=180.0,
                                deg_per_frame=0.5)[0]
    tables = adjoint.scene_tables(sc, iv, ip, W, H)
    plain = adjoint.AdjointRenderer(tables, spp=1, max_depth=8, seed=1, device=dev, miss_radiance=0.5)
    alb = torch.from_numpy(tables.albedo_target).to(dev)
    em = torch.from_numpy(tables.emission_target).to(dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, reps=1):
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record()
        for _ in range(reps):
            out = fn()
        b.record()
        torch.cuda.synchronize()
        return out, a.elapsed_time(b) / reps

    # reference: 4096 spp in 16 chunks of 256 with disjoint sample ids
    ref = torch.zeros((H, W, 3), dtype=torch.float64, device=dev)
    for k in range(16):
        plain.seed = 1000001 + 256 * k
        ref += plain.forward(alb, em, spp=256).double()
    ref /= 16.0

    def relmse(img):
        r = ref.float()
        return float((((img - r) ** 2) / (r * r + 1e-2)).mean())

    plain_rows = []
    for spp in (1, 2, 4, 8, 16, 32):
        plain.seed = 7 + 1000 * spp
        img, ms = timed(lambda: plain.forward(alb, em, spp=spp), reps=3)
        plain_rows.append((spp, relmse(img), ms))
    cache = nrc.NrcCache((0.0, 0.0, 0.0), (float(edge),) * 3, device=dev, lr=1e-3)
    nr = nrc.NrcRenderer(plain, cache, train_paths=1 << 16, train_bounces=4)
    losses = []
    clocks = ClockSampler(dev.index if dev.index is not None else 0).wait_ready()
    for f in range(args.warmup * 60):  # online training before the timed frames
        _, (loss, _) = nr.render(5000 + f)
        losses.append(loss)
    fallbacks_warm = nr.fallbacks
    torch.cuda.synchronize()
    # every timed frame's image is kept for the error, in memory allocated
    # beforehand (an allocation per frame would wait for the device)
    imgs = torch.empty((args.steps, H, W, 3), dtype=torch.float32, device=dev)
    a, b = ev(), ev()
    a.record()
    for k in range(args.steps):
        _, (loss, n_train) = nr.render(9000 + k, out=imgs[k])
    b.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    nrc_ms = a.elapsed_time(b) / args.steps
    nrc_err = float(np.mean([relmse(i) for i in imgs]))
    # where a cache frame's time goes, and the fused MLP against the tensor
    # cores' peak: the same steps as NrcRenderer.render, timed one by one
    phase = {"trace": 0.0, "train": 0.0, "infer": 0.0}
    for k in range(args.steps):
        e = [ev() for _ in range(4)]
        e[0].record()
        nr.trace(9500 + k)
        e[1].record()
        nr.train()
        e[2].record()
        rgb = cache.infer(nr.query)
        e[3].record()
        torch.cuda.synchronize()
        for j, key in enumerate(phase):
            phase[key] += e[j].elapsed_time(e[j + 1]) / args.steps
    mlp_flops = 2.0 * W * H * (nrc.IN * nrc.WIDTH + (nrc.HIDDEN - 1) * nrc.WIDTH * nrc.WIDTH + nrc.WIDTH * nrc.OUT)
    peak, peak_src = measured_peaks("bf16_tflops")
    mlp_tflops = mlp_flops / (phase["infer"] * 1e-3) / 1e12
    # the plain spp of equal relMSE (relMSE ~ c / spp^alpha, fitted in log-log)
    xs = np.log([r[0] for r in plain_rows])
    ys = np.log([r[1] for r in plain_rows])
    alpha, logc = np.polyfit(xs, ys, 1)
    spp_equal = float(math.exp((math.log(nrc_err) - logc) / alpha))
    ms_per_spp = float(np.polyfit([r[0] for r in plain_rows], [r[2] for r in plain_rows], 1)[0])
    ms_plain_equal = ms_per_spp * spp_equal
    assert nrc.status() == 0
    return {
        "metric": "neural radiance cache: ms/frame at the plain tracer's equal relMSE", "value": round(nrc_ms, 4),
        "unit": "ms/frame", "n_gpus": world, "steps": args.steps, "warmup": args.warmup * 60,
        "ms_per_step": round(nrc_ms, 4), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 tracing, bf16 MLP weights with fp32 accumulation",
        "data": "synthetic (seeded 512^3 heightfield terrain, orbit camera)",
        "config": {"workload": "nrc_terrain512_1080p", "voxels": sc.voxel_count, "resolution": [W, H],
                   "mlp": "256 (freq 16 bands, one-blob 32 bins, albedo) -> 64 x 5 ReLU -> RGB",
                   "train": "2^16 self-training paths x 4 bounces per frame; 4 Adam steps (lr 1e-3) on 2^14 of "
                            "their vertices",
                   "cache_vertex": "path vertex 2 (camera 0, primary hit 1): the first bounce hit",
                   "plain": "ct_adjoint_forward, depth 8, grey sky 0.5", "reference_spp": 4096},
        "nrc_relmse": round(nrc_err, 5), "plain": [[r[0], round(r[1], 5), round(r[2], 4)] for r in plain_rows],
        "plain_spp_at_equal_relmse": round(spp_equal, 3), "plain_ms_at_equal_relmse": round(ms_plain_equal, 4),
        "ratio_nrc_over_plain": round(nrc_ms / ms_plain_equal, 4) if ms_plain_equal > 0 else None,
        "phase_ms": {k: round(v, 4) for k, v in phase.items()},
        "roofline": {"bound": "tensor", "kernel": "k_nrc_mlp (encoding + 6 layers, one launch per frame)",
                     "achieved": round(mlp_tflops, 2), "peak": peak, "unit": "TFLOP/s",
                     "frac": round(mlp_tflops / peak, 4), "peak_source": peak_src,
                     "flops_per_launch": mlp_flops, "traffic": None,
                     "note": "infer time includes the encoding (sin/cos, exp) and the 48 B/query reads"},
        "training_loss": [round(float(v), 4) for v in losses[::30]] + [round(float(loss), 4)],
        "fallback_frames_warmup": fallbacks_warm, "fallback_frames_timed": nr.fallbacks - fallbacks_warm,
        "clocks": clk,
    }


def native_flag_count_rays():
    from cube_tracing import native
    return native.CT_PARAM_COUNT_RAYS


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--width", type=int, default=W_DEFAULT)
    ap.add_argument("--height", type=int, default=H_DEFAULT)
    ap.add_argument("--edge", type=int, default=256)
    ap.add_argument("--ref-rows", type=int, default=240)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="terrain256_1080p", choices=["terrain256_1080p", "views32", "nrc"])
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return 0
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload in ("views32", "nrc"):
        out = (run_views if args.workload == "views32" else run_nrc)(args, rank, world)
        if rank == 0:
            print(json.dumps(out))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    out = run_b200(args, rank, world)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            base, why = oracle_sample(args)
            out["cpu_baseline"] = ({k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
                                   if base else {"unavailable": why})
            out["fp64_error"] = fp64_error_line(args)
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
