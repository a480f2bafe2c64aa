"""The C++ host side (ct::Renderer, cube-tracing_b200/host) renders the same
frames as the Python one: the check program runs a camera path through it
and its last frame's image and per-pixel buffers are compared byte for byte
with cube_tracing.frame.Renderer's on the same scene, cameras and
ct_params."""
import os

import pytest

import hostcpp
from cases import build_case

CASES = ["grid16_pt", "instances16_pt", "grid16_materials_brdf_pt"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cpp_host_matches_python_host(name, tmp_path):
    import torch
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    py = Renderer(sc, W, H, **kw)
    for iv, ip in cams:
        img = py.render(iv, ip)
    torch.cuda.synchronize()
    params = type(py.params).from_buffer_copy(bytes(py.params))
    params.workspace_address = 0
    params.workspace_bytes = 0
    inp, outp = os.path.join(tmp_path, "in.bin"), os.path.join(tmp_path, "out.bin")
    hostcpp.write_input(inp, sc, W, H, cams, params, py.features, int(py.status_host[0]["max_depth"]), taa=py.taa)
    r = hostcpp.run(inp, outp)
    assert r.returncode == 0, r.stderr
    cpp = hostcpp.read_output(outp)
    assert cpp["image"].tobytes() == img.cpu().numpy().tobytes()
    for k in hostcpp.RESTIR_ORDER:
        assert cpp[k].tobytes() == py.buf[k].cpu().numpy().tobytes(), k
