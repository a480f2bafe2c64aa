"""A randomized parity sweep: 100 seeded random cases (tests/sweep.py:
scenes, instance transforms, light types, BRDF candidates, materials, DI or
DI + PT, TAA, time of day, an erase between frames), each rendered by the
CUDA path and the oracle, every frame compared under the bar of
test_gpu_parity."""
import pytest

import sweep
from cases import frame_keys
from test_gpu_parity import compare_frame, gpu_frame, ref_frame

SEEDS = range(9900, 10000)


@pytest.mark.gpu
def test_random_cases_match_oracle(oracle_lib):
    from cube_tracing.frame import Renderer
    failing = []
    for k in SEEDS:
        sc, W, H, cams, kw, edit = sweep.make_case(k)
        keys = frame_keys("x_pt" if kw.get("indirect") else "x")
        ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
        gpu = Renderer(sc, W, H, **kw)
        problems = []
        for f, (iv, ip) in enumerate(cams):
            if edit is not None and f == 2:
                ora.erase(*edit)
                gpu.erase(*edit)
            ro = ref_frame(ora, ora.render(iv, ip), keys)
            rg = gpu_frame(gpu, gpu.render(iv, ip), keys)
            problems += compare_frame(f"case {k} frame {f}", W, rg, ro)
        err = gpu.device_error()
        ora.close()
        if problems or err != (0, 0, 0):
            failing.append(f"case {k} ({W}x{H}, {kw}): error {err}; " + "; ".join(problems[:3]))
    assert not failing, "\n".join(failing)
