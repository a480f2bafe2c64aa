"""Parity at the reference's own voxel edge, 2^-5 (VOXEL_EXTENT in
shared.inl); the other parity cases use unit voxels.  The walk's grid
scaling, the voxel centres and the box tests all take the edge.  A 16^3
grid scaled to 0.5 units, DI + PT to depth 4 + TAA, three frames, against
the oracle built for that edge (oracle/_ref/libct_oracle_e5.so), under the
bar of test_gpu_parity.py."""
import numpy as np
import pytest

from cube_tracing import layouts as L
from cube_tracing import scenes
from test_gpu_parity import compare_frame, gpu_frame, ref_frame

E5 = 0.03125
KEYS = ["di", "intermediate_reservoir", "previous_reservoir", "velocity", "output_path_reservoir",
        "temporal_path_reservoir", "indirect_color"]


def e5_case():
    s = np.float32(E5)
    sc = scenes.random_grid_scene(16, 0.3, emissive_fraction=0.05, seed=3, voxel_extent=E5)
    pl = np.zeros(1, L.LIGHT)
    pl["position"] = (8.0 * s, 30.0 * s, 8.0 * s)
    pl["emissive"] = (0.2, 0.2, 0.2)
    pl["instance_id"] = L.MAX_INSTANCES
    pl["primitive_id"] = L.MAX_PRIMITIVES
    pl["type"] = L.LIGHT_POINT
    sc.point_lights = pl
    sc.light_config["point_light_count"] = 1
    W, H = 36, 28
    cams = scenes.camera_path("translate", 3, W, H, eye=(-4.0 * s, 8.0 * s, -4.0 * s), target=(8.0 * s, 8.0 * s, 8.0 * s),
                              step=(0.1 * s, 0.0, 0.0))
    return sc, W, H, cams, {"indirect": True, "max_depth": 4}


def test_e5_oracle_built_for_the_edge(oracle_lib):
    if not oracle_lib.available(extent=E5):
        pytest.fail("oracle library for VOXEL_EXTENT 2^-5 not built (make -C oracle)")
    assert oracle_lib.info(extent=E5).voxel_extent == np.float32(E5)
    assert oracle_lib.info().voxel_extent == 1.0


@pytest.mark.gpu
def test_gpu_matches_oracle_at_reference_voxel_edge(oracle_lib):
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = e5_case()
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    assert gpu.sb.accel.info().grid_exact == 1
    problems = []
    hits = 0
    for f, (iv, ip) in enumerate(cams):
        ro = ref_frame(ora, ora.render(iv, ip), KEYS)
        rg = gpu_frame(gpu, gpu.render(iv, ip), KEYS)
        assert gpu.device_error() == (0, 0, 0)
        hits += int((ro["di"]["distance"] > 0).sum())
        problems += compare_frame(f"e5 frame {f}", W, rg, ro)
    assert hits > W * H  # the grid fills part of every frame
    assert not problems, "\n".join(problems)
