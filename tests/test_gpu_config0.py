"""Parity on the small plain workload at its full size (64^3 grid, 256x256,
8 frames, max depth 4, ReSTIR DI and PT, TAA): every frame of the CUDA path
against the oracle, with the bar of test_gpu_parity (bit-exact ids,
reservoir samples and counts, path flags; radiance within RTOL).  Two
cases: "config0" with the reference's compiled-in reuse parameters (3-4
neighbours in 2-50 px) and a point light, and "config0_spec" as the
workload is specified: 5 neighbours in a 30-pixel radius, no point light."""
import pytest

from cases import build_case, frame_keys
from test_gpu_parity import compare_frame, gpu_frame, ref_frame


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["config0", "config0_spec"])
def test_config0_all_frames_match_oracle(oracle_lib, name):
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    keys = frame_keys(name) + ["output_path_reservoir", "temporal_path_reservoir", "indirect_color"]
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    problems = []
    for f, (iv, ip) in enumerate(cams):
        ro = ref_frame(ora, ora.render(iv, ip), keys)
        rg = gpu_frame(gpu, gpu.render(iv, ip), keys)
        assert gpu.device_error() == (0, 0, 0)
        problems += compare_frame(f"{name} frame {f}", W, rg, ro)
    assert not problems, "\n".join(problems[:40])
