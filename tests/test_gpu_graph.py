"""Renderer.render_graph: frames replayed from CUDA graphs match frames
recorded launch by launch, bit for bit, across both output images, an edit
and the frames after it."""
import numpy as np
import pytest

from cases import build_case, frame_keys


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["grid16", "grid16_pt"])
def test_graph_frames_match_recorded_frames(name):
    import torch
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    a = Renderer(sc, W, H, **kw)
    b = Renderer(sc, W, H, **kw)
    keys = frame_keys(name)
    seq = list(cams) + list(cams[::-1])
    for f, (iv, ip) in enumerate(seq):
        if f == 4:
            assert len(b._graphs) == 2  # one per output image
            a.erase((W // 2, H // 2), 3)
            b.erase((W // 2, H // 2), 3)
        ia = a.render(iv, ip).cpu().numpy()
        ib = b.render_graph(iv, ip).cpu().numpy()
        torch.cuda.synchronize()
        assert np.array_equal(ia, ib), f"frame {f} image"
        for k in keys:
            assert a.read(k).tobytes() == b.read(k).tobytes(), f"frame {f} {k}"
    assert a.device_error() == (0, 0, 0) and b.device_error() == (0, 0, 0)
