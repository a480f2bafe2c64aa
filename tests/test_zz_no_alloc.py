"""ct_restir_di_static (library-resident scratch, no allocation) against
ct_restir_di (caller or library-allocated workspace), through the C ABI.

Both renderers share one scene and acceleration structure and render the same
two-frame camera path; every per-pixel buffer and the output image must agree
within RTOL after each of the two calls in a row.  A frame whose scratch
exceeds CT_STATIC_WORKSPACE_BYTES must be refused with CT_ERR_CAPACITY.
"""
import ctypes

import numpy as np
import pytest

from cases import FRAME_KEYS, build_case

pytestmark = pytest.mark.gpu

RTOL = 1e-4
ATOL = 1e-6
CT_ERR_CAPACITY = 2
STATIC_BYTES = 40 << 20


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _render_static(r, inv_view, inv_proj):
    """Renderer.render with ct_restir_di replaced by ct_restir_di_static."""
    import torch
    from cube_tracing import layouts as L
    from cube_tracing import native
    is_active = r._upload(inv_view, inv_proj)
    pc = r.push_constant()
    stream = torch.cuda.current_stream().cuda_stream
    lib = native.lib()
    p = ctypes.byref(r.params)
    native.check("ct_trace_frame", lib.ct_trace_frame(ctypes.byref(pc), p, stream))
    native.check("ct_restir_di_static", lib.ct_restir_di_static(ctypes.byref(pc), p, 0, stream))
    native.check("ct_restir_di_static", lib.ct_restir_di_static(ctypes.byref(pc), p, 1, stream))
    if is_active & L.TAA_BIT:
        native.check("ct_taa", lib.ct_taa(ctypes.byref(pc), p, stream))
    out = r.images[r.frame % 2]
    r.prev_cam = (np.array(inv_view), np.array(inv_proj))
    r.frame += 1
    return out


def _close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return (np.isnan(a) & np.isnan(b)) | (np.abs(a - b) <= RTOL * np.maximum(np.abs(a), np.abs(b)) + ATOL)


def _compare(tag, ref, got):
    for key in FRAME_KEYS:
        a, b = ref.read(key), got.read(key)
        for f in a.dtype.names:
            assert _close(a[f], b[f]).all(), f"{tag}: {key}.{f} differs"


@pytest.mark.parametrize("case,size", [("grid32_allfeatures", None), ("terrain32", (256, 144))])
def test_static_matches_allocating_entry_point(case, size):
    torch = _torch()
    from cube_tracing import frame, native, scenes
    sc, W, H, cams, kw = build_case(case)
    if size is not None:
        W, H = size
        cams = scenes.camera_path("orbit", 2, W, H, center=(16.0, 8.0, 16.0), radius=40.0, elevation=25.0,
                                  deg_per_frame=1.0)
    need = ctypes.c_uint64()
    native.check("ct_workspace_size", native.lib().ct_workspace_size(W, H, native.params_for_scene(sc),
                                                                     ctypes.byref(need)))
    assert need.value <= STATIC_BYTES
    sb = frame.SceneBuffers(sc)
    ref = frame.Renderer(sc, W, H, scene_buffers=sb, **kw)
    got = frame.Renderer(sc, W, H, scene_buffers=sb, **kw)
    for i, (iv, ip) in enumerate(cams[:2]):
        a = ref.render(iv, ip, stages=("trace", "di0", "di1", "taa"))
        b = _render_static(got, iv, ip)
        torch.cuda.synchronize()
        assert got.device_error() == (0, 0, 0)
        assert _close(a.cpu().numpy(), b.cpu().numpy()).all(), f"{case} call {i}: image differs"
        _compare(f"{case} call {i}", ref, got)


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
