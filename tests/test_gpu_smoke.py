"""The build entry's smoke run (a small DI + PT frame sequence on cuda:0
against the oracle) stays runnable."""
import pytest


@pytest.mark.gpu
def test_smoke():
    import __graft_entry__
    __graft_entry__.smoke()


@pytest.mark.gpu
def test_walk_cap_latches_iteration_limit_and_the_context_stays_usable(oracle_lib):
    """Failure path of the walk's iteration cap (CT_ERR_ITER_LIMIT), made to
    happen by a tiny ct_params.walk_step_limit instead of by a fault: the
    frame ends, the status word holds the error and a pixel, and the next
    frames with the normal cap render without error and match the oracle."""
    from cases import build_case, frame_keys
    from cube_tracing.frame import Renderer
    from test_gpu_parity import compare_frame, gpu_frame, ref_frame
    name = "grid16_pt"
    sc, W, H, cams, kw = build_case(name)
    capped = Renderer(sc, W, H, **kw)
    capped.params.walk_step_limit = 2
    capped.render(*cams[0])
    status, detail, pixel = capped.device_error()
    assert status == 4 and pixel < W * H, (status, detail, pixel)
    assert capped.device_error() == (0, 0, 0)  # read and reset
    gpu = Renderer(sc, W, H, **kw)
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    problems = []
    for f, (iv, ip) in enumerate(cams):
        rg = gpu_frame(gpu, gpu.render(iv, ip), frame_keys(name))
        ro = ref_frame(ora, ora.render(iv, ip), frame_keys(name))
        problems += compare_frame(f"after the cap, frame {f}", W, rg, ro)
    assert gpu.device_error() == (0, 0, 0)
    assert not problems, "\n".join(problems)
    ora.close()
