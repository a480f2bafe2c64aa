"""Many views rendered side by side (ct_render_views, cube_tracing.views):
every view of a batch replayed from a CUDA graph against the oracle, the
batch against the same views rendered one after another, and the
schedule autotuner.

The workload is the many-view kind at test size: seeded random grids with
edge and occupancy drawn per scene, views of drawn resolutions on them
(odd sizes, so TAA's edge rule is exercised), DI with one temporal and one
spatial pass, ReSTIR PT to depth 6, TAA."""
import numpy as np
import pytest

from cases import FRAME_KEYS, PT_KEYS
from test_gpu_parity import compare_frame, gpu_frame, ref_frame

pytestmark = pytest.mark.gpu

KW = {"indirect": True, "max_depth": 6}


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def _small():
    from cube_tracing import views
    return views.views_workload(n_scenes=3, n_views=6, seed=7, edge_range=(12, 24), res_min=(16, 12),
                                res_max=(48, 40))


def test_batched_views_match_oracle(oracle_lib):
    torch = _torch()
    from cube_tracing import views
    scs, vs = _small()
    mv = views.MultiViewRenderer(scs, vs, **KW)
    mv.set_schedule(lanes=4, walker="proportional")
    oras = [oracle_lib.OracleRenderer(scs[v["scene"]], v["width"], v["height"], **KW) for v in vs]
    keys = FRAME_KEYS + PT_KEYS
    problems = []
    for f in range(3):
        cams = mv.cams(f)
        mv.render(cams)
        torch.cuda.synchronize()
        assert mv.device_error() == (0, 0, 0)
        for i, (r, o) in enumerate(zip(mv.r, oras)):
            rg = gpu_frame(r, r.images[f % 2], keys)
            ro = ref_frame(o, o.render(*cams[i]), keys)
            problems += compare_frame(f"view {i} ({r.W}x{r.H}) frame {f}", r.W, rg, ro)
    for o in oras:
        o.close()
    assert not problems, "\n".join(problems[:40])


def test_batch_equals_views_rendered_one_by_one():
    torch = _torch()
    from cube_tracing import views
    scs, vs = views.views_workload(n_scenes=4, n_views=8, seed=11, edge_range=(24, 64), res_min=(40, 32),
                                   res_max=(256, 192))
    a = views.MultiViewRenderer(scs, vs, **KW)
    b = views.MultiViewRenderer(scs, vs, **KW)
    a.set_schedule(lanes=8, walker="proportional")
    for f in range(4):
        a.render(a.cams(f))
        b.render_sequential(b.cams(f))
    torch.cuda.synchronize()
    for i, (ra, rb) in enumerate(zip(a.r, b.r)):
        assert np.array_equal(ra.images[0].cpu().numpy().view(np.uint32), rb.images[0].cpu().numpy().view(np.uint32)), i
        assert np.array_equal(ra.images[1].cpu().numpy().view(np.uint32), rb.images[1].cpu().numpy().view(np.uint32)), i
        for k in FRAME_KEYS + PT_KEYS:
            assert np.array_equal(ra.buf[k].cpu().numpy(), rb.buf[k].cpu().numpy()), (i, k)


def test_autotune_keeps_the_fastest_schedule():
    _torch()
    from cube_tracing import views
    scs, vs = _small()
    mv = views.MultiViewRenderer(scs, vs, **KW)
    table = mv.autotune(lanes_options=(0, 2, 6), frames=2)
    assert len(table) == 6
    assert [t[2] for t in table] == sorted(t[2] for t in table)
    assert mv.schedule == {"lanes": table[0][0], "walker": table[0][1]}
    assert all(t[2] > 0 for t in table)
