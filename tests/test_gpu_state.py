"""Frame history checkpoint on the GPU: a renderer that loads the state
saved after frame k continues the run exactly, and the same blob moves a
run between the CUDA path and the oracle in either direction, so that a
parity check can start both from identical state at any frame."""
import numpy as np
import pytest

from cases import build_case, frame_keys
from test_gpu_parity import compare_frame, gpu_frame, ref_frame

CASES = ["grid16_pt", "grid16_materials_brdf_pt", "instances16"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_resumes_from_saved_state(name):
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    keys = frame_keys(name)
    a = Renderer(sc, W, H, **kw)
    for iv, ip in cams[:2]:
        a.render(iv, ip)
    state = a.save_state()
    b = Renderer(sc, W, H, **kw)
    b.load_state(state)
    ra = gpu_frame(a, a.render(*cams[2]), keys)
    rb = gpu_frame(b, b.render(*cams[2]), keys)
    assert ra["image"].tobytes() == rb["image"].tobytes()
    for k in keys:
        assert ra[k].tobytes() == rb[k].tobytes(), k
    assert a.device_error() == (0, 0, 0) and b.device_error() == (0, 0, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("direction", ["gpu_to_oracle", "oracle_to_gpu"])
def test_state_moves_between_gpu_and_oracle(oracle_lib, name, direction):
    """Two frames on one side, the saved history loaded into the other, and
    the third frame rendered by both from that one state."""
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    keys = frame_keys(name)
    gpu = Renderer(sc, W, H, **kw)
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    src, dst = (gpu, ora) if direction == "gpu_to_oracle" else (ora, gpu)
    for iv, ip in cams[:2]:
        src.render(iv, ip)
    state = src.save_state()
    dst.load_state(state)
    assert gpu.frame == ora.frame == 2
    rg = gpu_frame(gpu, gpu.render(*cams[2]), keys)
    ro = ref_frame(ora, ora.render(*cams[2]), keys)
    assert gpu.device_error() == (0, 0, 0)
    problems = compare_frame(f"{name} {direction} frame 2", W, rg, ro)
    assert not problems, "\n".join(problems)
    ora.close()


@pytest.mark.gpu
def test_load_rejects_a_state_of_another_size():
    import ctypes
    from cube_tracing import native
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case("grid16_pt")
    a = Renderer(sc, W, H, **kw)
    a.render(*cams[0])
    blob, frame, prev = a.save_state()
    small = Renderer(sc, W // 2, H, **kw)
    small.render(*cams[0])
    pc = small.push_constant()
    bad = np.ascontiguousarray(blob)
    assert native.lib().ct_state_load(ctypes.byref(pc), bad.ctypes.data, bad.size, None) == 1
    # the right size with another frame's header
    n = small.state_size()
    fake = np.zeros(n, np.uint8)
    fake[:blob.size if blob.size < n else n] = blob[:min(n, blob.size)]
    assert native.lib().ct_state_load(ctypes.byref(pc), fake.ctypes.data, fake.size, None) == 1
