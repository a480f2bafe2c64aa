"""The sun and day/night cycle helper against the reference host's formulas
(src/main.cpp:180-232, 440-444, 497-510), and (GPU) frames under a moving sun
against the oracle."""
import numpy as np
import pytest

from cube_tracing import daylight as D
from cube_tracing import layouts as L


def test_sun_positions_and_intensity():
    assert np.array_equal(D.sun_position(1.0, True), D.SUN_TOP_POSITION)
    assert np.array_equal(D.sun_position(0.0, True), D.SUNSET_POSITION)
    assert np.array_equal(D.sun_position(0.0, False), -D.SUNSET_POSITION)
    np.testing.assert_allclose(D.sun_position(0.5, True), [10.0, 7.5, -2.5])
    assert D.sun_intensity(0.49, True) == 0.0
    assert D.sun_intensity(0.5, True) == np.float32(5000.0)
    assert D.sun_intensity(1.0, False) == D.SUN_MAX_INTENSITY


def test_cycle_flips_at_the_ends():
    pl, t, aft = D.make_sun()
    t = D.add_time(t, aft, 0.25)              # past midday in the afternoon
    t, aft = D.update_sun(t, aft, pl)
    assert (t, aft) == (np.float32(1.0), False)
    t = D.add_time(t, aft, 0.25)              # the morning runs backwards
    t, aft = D.update_sun(t, aft, pl)
    assert t == np.float32(0.75) and aft is False
    np.testing.assert_allclose(pl[0]["position"], D.sun_position(0.75, False))
    assert pl[0]["emissive"][0] == np.float32(7500.0)


@pytest.mark.gpu
def test_frames_under_a_moving_sun_match_oracle(oracle_lib):
    from cases import build_case, frame_keys
    from cube_tracing.frame import Renderer
    from test_gpu_parity import compare_frame, gpu_frame, ref_frame
    sc, W, H, cams, kw = build_case("grid32_allfeatures_pt")
    sun, t, aft = D.make_sun()
    sc.point_lights = sun
    t, aft = np.float32(0.55), False
    ora = oracle_lib.OracleRenderer(sc, W, H, sky_time=float(t), is_afternoon=int(aft), **kw)
    gpu = Renderer(sc, W, H, sky_time=float(t), is_afternoon=int(aft), **kw)
    keys = frame_keys("grid32_allfeatures_pt")
    problems = []
    for f in range(4):
        iv, ip = cams[min(f, len(cams) - 1)]
        t, aft = D.update_sun(t, aft, sun)
        ora.set_point_lights(sun)
        gpu.sb.set_point_lights(sun)
        ora.set_time(t, aft)
        gpu.set_time(t, aft)
        ro = ref_frame(ora, ora.render(iv, ip), keys)
        rg = gpu_frame(gpu, gpu.render(iv, ip), keys)
        assert gpu.device_error() == (0, 0, 0)
        problems += compare_frame(f"sun t={t} afternoon={aft} frame {f}", W, rg, ro)
        t = D.add_time(t, aft, 0.2)
    assert not problems, "\n".join(problems[:40])
