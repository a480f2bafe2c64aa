"""Parity on the benchmark's own workload: the 256^3 heightfield terrain at
1920x1080 with the benchmark's parameters (32 cube-light candidates,
temporal reuse and 2 DI spatial rounds, ReSTIR PT to depth 8 with the
hybrid shift and temporal and spatial path reuse, TAA keeping 0.9 of the
history), three frames of
the orbit rendered whole by the CUDA path and by the oracle (the
reference's shaders with the same run-time parameters), with the bar of
test_gpu_parity: bit-exact ids, reservoir samples and counts and path
flags; radiance within RTOL.

A second test states the error of the CUDA frame itself against the FP64
build of the oracle: the oracle continues the CUDA run from its saved
history (ct_state_save) and renders the next frame over a band of rows with
a margin wider than the frame's reach across rows (two spatial rounds of at
most 50 px, TAA's 3x3 window), so that the band's pixels see the same
inputs as in the full frame."""
import numpy as np
import pytest

from cases import FRAME_KEYS, PT_KEYS
from test_gpu_parity import compare_frame, gpu_frame, ref_frame

pytestmark = pytest.mark.gpu


def _workload():
    import bench
    sc = bench.workload(256)
    W, H = bench.W_DEFAULT, bench.H_DEFAULT
    return bench, sc, W, H


def test_headline_frames_match_oracle(oracle_lib):
    from cube_tracing.frame import Renderer
    bench, sc, W, H = _workload()
    cams = bench.camera_frames(3, W, H)
    kw = {"indirect": True, "max_depth": bench.MAX_DEPTH, "params": bench.headline_params()}
    keys = FRAME_KEYS + PT_KEYS
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    assert gpu.params.spatial_passes == 2 and abs(gpu.params.taa_alpha - 0.1) < 1e-7
    assert gpu.params.pt_shift_mapping == 2 and gpu.params.pt_near_field_distance == 0.5
    problems = []
    for f, (iv, ip) in enumerate(cams):
        rg = gpu_frame(gpu, gpu.render(iv, ip), keys)
        assert gpu.device_error() == (0, 0, 0)
        ro = ref_frame(ora, ora.render(iv, ip), keys)
        problems += compare_frame(f"terrain256 1080p frame {f}", W, rg, ro)
        hit = ro["di"]["distance"] > 0
        assert 0.3 < hit.mean() < 1.0  # the frame shows terrain and sky
    ora.close()
    assert not problems, "\n".join(problems[:40])


def test_headline_cuda_frame_error_against_fp64(oracle_lib):
    import torch
    from cube_tracing.frame import Renderer
    if not oracle_lib.available(fp64=True):
        pytest.fail("FP64 oracle not built (make -C oracle)")
    bench, sc, W, H = _workload()
    cams = bench.camera_frames(3, W, H)
    kw = {"indirect": True, "max_depth": bench.MAX_DEPTH, "params": bench.headline_params()}
    gpu = Renderer(sc, W, H, **kw)
    err = bench.cuda_fp64_error(gpu, sc, W, H, cams, band=(480, 560), threads=0)
    torch.cuda.synchronize()
    # choices agree on almost every hit pixel; where they agree the image is
    # within a few ulps of FP32
    assert err["ids_equal"] > 0.999
    assert err["reservoirs_equal"] > 0.99
    assert err["paths_equal"] > 0.99
    assert err["image_rel_err"]["median"] < 1e-5
    assert err["image_rel_err"]["p99"] < 1e-3
    assert np.isfinite(err["image_rel_err_all"]["max"])
