"""ct_restir_di_static (library-resident scratch, no allocation) against
ct_restir_di (caller or library-allocated workspace), through the C ABI.

Some hosts cannot allocate device memory while they render: engines that
hand out memory only from an arena reserved at start-up, or plug-in hosts
that own every allocation.  ct_restir_di_static serves them with scratch
compiled into the library.  It runs the same kernels on the same inputs as
ct_restir_di, so every per-pixel buffer and the output image must be equal
bit for bit after each of two calls in a row, in every case below:

  * default parameters (two scenes, one of them at 256x144);
  * a walk cap of a few cells (ct_params.walk_step_limit): both entry points
    must latch CT_ERR_ITER_LIMIT and leave the same frame;
  * three spatial rounds (the intermediate/current ping-pong);
  * the frame after a scene edit (tlas_previous bound, REMAP_BIT set);
  * ReSTIR PT on (CT_PARAM_INDIRECT): ct_restir_pt keeps its own workspace
    between the two static DI stages.

A frame whose scratch exceeds CT_STATIC_WORKSPACE_BYTES must be refused with
CT_ERR_CAPACITY.  This file is collected last, so that a run stopping at the
first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

from cases import FRAME_KEYS, PT_KEYS, build_case

pytestmark = pytest.mark.gpu

CT_ERR_CAPACITY = 2
CT_ERR_ITER_LIMIT = 4
STATIC_BYTES = 40 << 20


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _render_static(r, inv_view, inv_proj):
    """Renderer.render with ct_restir_di replaced by ct_restir_di_static
    (ct_restir_pt, when the frame has it, keeps the renderer's workspace)."""
    import torch
    from cube_tracing import layouts as L
    from cube_tracing import native
    is_active = r._upload(inv_view, inv_proj)
    pc = r.push_constant()
    stream = torch.cuda.current_stream().cuda_stream
    lib = native.lib()
    p = ctypes.byref(r.params)
    indirect = bool(r.params.flags & native.CT_PARAM_INDIRECT)
    native.check("ct_trace_frame", lib.ct_trace_frame(ctypes.byref(pc), p, stream))
    native.check("ct_restir_di_static", lib.ct_restir_di_static(ctypes.byref(pc), p, 0, stream))
    if indirect:
        native.check("ct_restir_pt", lib.ct_restir_pt(ctypes.byref(pc), p, 0, stream))
    native.check("ct_restir_di_static", lib.ct_restir_di_static(ctypes.byref(pc), p, 1, stream))
    if indirect:
        native.check("ct_restir_pt", lib.ct_restir_pt(ctypes.byref(pc), p, 1, stream))
    if is_active & L.TAA_BIT:
        native.check("ct_taa", lib.ct_taa(ctypes.byref(pc), p, stream))
    out = r.images[r.frame % 2]
    r.prev_cam = (np.array(inv_view), np.array(inv_proj))
    r.frame += 1
    if r.sb.accel_prev is not None:
        # the settling step Renderer.render takes after an edit frame
        r.sb.remap_p.zero_()
        r.sb.remap_l.zero_()
        r.sb.accel_retired.append(r.sb.accel_prev)
        r.sb.accel_prev = None
    return out


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def _compare(tag, ref, got, keys):
    for key in keys:
        a, b = ref.read(key), got.read(key)
        for f in a.dtype.names or [None]:
            x, y = (a, b) if f is None else (a[f], b[f])
            assert np.array_equal(_bits(x), _bits(y)), f"{tag}: {key}.{f or ''} differs"


CASES = {
    # name: (scene case, frame size or None, parameter overrides, edit before the second frame)
    "grid32_allfeatures": ("grid32_allfeatures", None, {}, False),
    "terrain32_256x144": ("terrain32", (256, 144), {}, False),
    "walk_cap": ("terrain32", None, {"walk_step_limit": 3}, False),
    "three_spatial_rounds": ("grid16", None, {"spatial_passes": 3}, False),
    "after_edit": ("grid16", None, {}, True),
    "with_pt": ("grid16_pt", None, {}, False),
}


@pytest.mark.parametrize("name", list(CASES))
def test_static_matches_allocating_entry_point(name):
    torch = _torch()
    from cube_tracing import frame, native, scenes
    case, size, overrides, edit = CASES[name]
    sc, W, H, cams, kw = build_case(case)
    if size is not None:
        W, H = size
        cams = scenes.camera_path("orbit", 2, W, H, center=(16.0, 8.0, 16.0), radius=40.0, elevation=25.0,
                                  deg_per_frame=1.0)
    need = ctypes.c_uint64()
    native.check("ct_workspace_size", native.lib().ct_workspace_size(
        W, H, native.params_for_scene(sc, **overrides), ctypes.byref(need)))
    assert need.value <= STATIC_BYTES
    # separate scene buffers, so that an edit changes each side's own scene
    ref = frame.Renderer(sc, W, H, params=native.params_for_scene(sc, **overrides), **kw)
    got = frame.Renderer(sc, W, H, params=native.params_for_scene(sc, **overrides), **kw)
    keys = FRAME_KEYS + (PT_KEYS if kw.get("indirect") else [])
    capped = overrides.get("walk_step_limit", 0) != 0
    for i, (iv, ip) in enumerate(cams[:2]):
        if edit and i == 1:
            for r in (ref, got):
                r.erase((18, 14), window=4)
        a = ref.render(iv, ip)
        e_ref = ref.device_error()
        b = _render_static(got, iv, ip)
        torch.cuda.synchronize()
        e_got = got.device_error()
        if capped:
            assert e_ref[0] == CT_ERR_ITER_LIMIT, e_ref
            assert e_got[0] == CT_ERR_ITER_LIMIT, e_got
        else:
            assert e_ref == (0, 0, 0) and e_got == (0, 0, 0), (e_ref, e_got)
        assert np.array_equal(_bits(a.cpu().numpy()), _bits(b.cpu().numpy())), f"{name} call {i}: image differs"
        _compare(f"{name} call {i}", ref, got, keys)


def test_static_rejects_frames_beyond_its_scratch():
    _torch()
    from cube_tracing import frame, native
    sc, W, H, cams, kw = build_case("terrain32")
    W, H = 1024, 1024
    need = ctypes.c_uint64()
    native.check("ct_workspace_size", native.lib().ct_workspace_size(W, H, native.params_for_scene(sc),
                                                                     ctypes.byref(need)))
    assert need.value > STATIC_BYTES
    r = frame.Renderer(sc, W, H, **kw)
    r._upload(*cams[0])
    pc = r.push_constant()
    for stage in (0, 1):
        st = native.lib().ct_restir_di_static(ctypes.byref(pc), ctypes.byref(r.params), stage, 0)
        assert st == CT_ERR_CAPACITY
