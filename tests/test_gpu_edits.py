"""Scene edits on the GPU (ct_brush, ct_rearrange, rebuild) against the CPU
restatement (oracle/edits.py), and the frames after an edit -- rendered
with REMAP_BIT against the previous scene -- against the oracle running the
reference's shaders.  Bit-exact for every id, count and table; the frames
use the parity bar of test_gpu_parity."""
import numpy as np
import pytest

import edits
from cases import build_case, frame_keys
from cube_tracing import layouts as L
from test_gpu_parity import compare_frame, gpu_frame, ref_frame

EDIT_CASES = [
    # (case, brush pixel, half window)
    ("grid16", (18, 14), 4),
    ("vox_room_pt", (20, 16), 5),
    ("terrain32", (16, 20), 6),
]


def _same(a, b):
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("name,pixel,window", EDIT_CASES)
def test_brush_and_rearrange_match_restatement(name, pixel, window):
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    r = Renderer(sc, W, H, **kw)
    for iv, ip in cams[:2]:
        r.render(iv, ip)
    before = r.scene_state()
    prev_di = r.read("previous_di")
    r.brush(pixel, window)
    marked = r.scene_state()
    want_p, want_i = edits.brush(prev_di, W, H, pixel, window, before["instances"])
    assert want_p.size > 0
    bits = np.unpackbits(marked["primitive_bitmask"].view(np.uint8), bitorder="little")
    assert np.nonzero(bits)[0].tolist() == want_p.tolist()
    ibits = np.unpackbits(marked["instance_bitmask"].view(np.uint8), bitorder="little")
    assert np.nonzero(ibits)[0].tolist() == want_i.tolist()
    assert marked["brush_counter"].tolist() == [want_i.size, want_p.size]

    r.rearrange()
    got = r.scene_state()
    ref = {k: v.copy() for k, v in before.items()}
    edits.rearrange(ref["instances"], ref["primitives"], ref["aabbs"], ref["cube_lights"], ref["light_config"],
                    want_p, want_i, ref["remap_p"], ref["remap_l"])
    for k in ("instances", "primitives", "aabbs", "cube_lights", "light_config", "remap_p", "remap_l"):
        assert _same(got[k], ref[k]), k
    assert not got["primitive_bitmask"].any() and not got["instance_bitmask"].any()
    assert not got["brush_counter"].any()
    assert r.device_error() == (0, 0, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("name,pixel,window", EDIT_CASES)
def test_frames_after_an_edit_match_oracle(oracle_lib, name, pixel, window):
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    keys = frame_keys(name)
    problems = []
    # two frames, the edit, then frames with REMAP_BIT (first) and without
    frames = list(cams) + [cams[-1]]
    for f, (iv, ip) in enumerate(frames):
        if f == 2:
            marks = ora.erase(pixel, window)
            gpu.erase(pixel, window)
            st = gpu.scene_state()
            assert marks[0].size > 0
            assert _same(st["instances"], ora._keep[0]) and _same(st["primitives"], ora._keep[1])
            assert _same(st["remap_p"], ora._keep[7][:st["remap_p"].shape[0]])
            assert _same(st["light_config"], ora.light_config)
        ro = ref_frame(ora, ora.render(iv, ip), keys)
        rg = gpu_frame(gpu, gpu.render(iv, ip), keys)
        assert gpu.device_error() == (0, 0, 0)
        problems += compare_frame(f"{name} frame {f}", W, rg, ro)
    assert not problems, "\n".join(problems)
    ora.close()


@pytest.mark.gpu
def test_removing_a_whole_instance_and_part_of_another(oracle_lib):
    """Marks written straight into the bitmasks: every primitive of the .vox
    room's second model and every third one of the first.  The
    rearrangement handles both instances in one call, the second instance is
    left empty, and the frames after it still match the oracle."""
    import torch
    from cube_tracing.frame import Renderer
    name = "vox_room_pt"
    sc, W, H, cams, kw = build_case(name)
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    keys = frame_keys(name)
    inst = sc.instances
    f1, n1 = int(inst["first_primitive_index"][1]), int(inst["primitive_count"][1])
    marked = np.concatenate([np.arange(0, int(inst["primitive_count"][0]), 3), np.arange(f1, f1 + n1)])
    frames = list(cams) + [cams[-1]]
    problems = []
    for f, (iv, ip) in enumerate(frames):
        if f == 2:
            bits = np.zeros(gpu.sb.primitive_bitmask.numel() * 32, np.uint8)
            bits[marked] = 1
            words = np.packbits(bits, bitorder="little").view(np.int32)
            gpu.sb.primitive_bitmask.copy_(torch.from_numpy(words.copy()).to(gpu.sb.primitive_bitmask.device))
            gpu.sb.instance_bitmask.fill_(0)
            gpu.sb.instance_bitmask[0] = 3  # instances 0 and 1
            gpu.sb.brush_counter.copy_(torch.tensor([2, marked.size], dtype=torch.int32))
            gpu.rearrange()
            gpu.rebuild()
            ora.remove(marked, [0, 1])
            st = gpu.scene_state()
            assert st["instances"]["primitive_count"][1] == 0
            for k, o in (("instances", ora._keep[0]), ("primitives", ora._keep[1]), ("aabbs", ora._keep[2]),
                         ("light_config", ora.light_config)):
                assert _same(st[k], o), k
            assert _same(st["remap_p"], ora._keep[7][:st["remap_p"].shape[0]])
        ro = ref_frame(ora, ora.render(iv, ip), keys)
        rg = gpu_frame(gpu, gpu.render(iv, ip), keys)
        assert gpu.device_error() == (0, 0, 0)
        problems += compare_frame(f"{name} frame {f}", W, rg, ro)
    assert not problems, "\n".join(problems)
    ora.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,pixel,window", EDIT_CASES)
def test_accel_voxel_count_follows_an_edit(name, pixel, window):
    """ct_accel_get_info's voxel count is the scene's distinct voxels, and
    after an erase the rebuilt structure holds exactly the removed ones fewer."""
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    r = Renderer(sc, W, H, **kw)
    distinct = sum(np.unique(sc.aabbs["minimum"][int(i["first_primitive_index"]):
                                                 int(i["first_primitive_index"]) + int(i["primitive_count"])],
                             axis=0).shape[0] for i in sc.instances)
    assert r.sb.accel.info().voxel_count == distinct
    for iv, ip in cams[:2]:
        r.render(iv, ip)
    marked, _ = edits.brush(r.read("previous_di"), W, H, pixel, window, sc.instances)
    r.erase(pixel, window)
    assert r.sb.accel.info().voxel_count == distinct - marked.size
