"""Scene edits on the CPU: known answers of the restated brush and
rearrangement (oracle/edits.py, squared_brush.slang / rearrangement.slang),
and the oracle's frame after an edit (REMAP_BIT, previous scene)."""
import numpy as np

import edits
from cases import build_case
from cube_tracing import layouts as L


def _scene(n_inst_prims, lights_at=()):
    """Instances of the given primitive counts on consecutive ranges, one
    voxel per primitive along x; cube lights on the listed global primitives."""
    insts = np.zeros(len(n_inst_prims), L.INSTANCE)
    first = 0
    for i, n in enumerate(n_inst_prims):
        insts[i]["first_primitive_index"] = first
        insts[i]["primitive_count"] = n
        first += n
    prims = np.zeros(first, L.PRIMITIVE)
    prims["material_index"] = np.arange(first)
    prims["light_index"] = 0xFFFFFFFF
    aabbs = np.zeros(first, L.AABB)
    aabbs["minimum"][:, 0] = np.arange(first)
    aabbs["maximum"] = aabbs["minimum"] + 1
    lights = np.zeros(len(lights_at), L.LIGHT)
    for li, g in enumerate(lights_at):
        i = int(np.searchsorted(np.cumsum(n_inst_prims), g, side="right"))
        lights[li]["instance_id"] = i
        lights[li]["primitive_id"] = g - insts[i]["first_primitive_index"]
        lights[li]["position"] = (g + 0.5, 0.5, 0.5)
        lights[li]["type"] = L.LIGHT_CUBE
        prims[g]["light_index"] = li
    cfg = np.zeros(1, L.LIGHT_CONFIG)
    cfg["cube_light_count"] = len(lights_at)
    cfg["light_count"] = len(lights_at) + 1
    return insts, prims, aabbs, lights, cfg


def test_rearrange_single_primitive_is_swap_with_last():
    insts, prims, aabbs, lights, cfg = _scene([8])
    rp, rl = np.zeros(8, np.uint32), np.zeros(1, np.uint32)
    edits.rearrange(insts, prims, aabbs, lights, cfg, [2], [0], rp, rl)
    assert insts["primitive_count"][0] == 7
    assert prims["material_index"][2] == 7 and aabbs["minimum"][2, 0] == 7
    assert rp.tolist() == [0, 0, 0xFFFFFFFF, 0, 0, 0, 0, 2]


def test_rearrange_pairs_in_rank_order():
    # 10 primitives, marks {1, 3, 8}: n2 = 7, head marks [1, 3] take the
    # unmarked tail [7, 9]; 8 is removed in place
    insts, prims, aabbs, lights, cfg = _scene([10])
    rp, rl = np.zeros(10, np.uint32), np.zeros(1, np.uint32)
    edits.rearrange(insts, prims, aabbs, lights, cfg, [1, 3, 8], [0], rp, rl)
    assert insts["primitive_count"][0] == 7
    assert prims["material_index"][:7].tolist() == [0, 7, 2, 9, 4, 5, 6]
    assert rp[[1, 3, 8]].tolist() == [0xFFFFFFFF] * 3
    assert rp[7] == 1 and rp[9] == 3
    assert rp[[0, 2, 4, 5, 6]].tolist() == [0] * 5


def test_rearrange_lights_follow_and_compact():
    # instance 0: 6 primitives, instance 1: 4; lights on 1, 4, 5 (inst 0) and 7 (inst 1)
    insts, prims, aabbs, lights, cfg = _scene([6, 4], lights_at=[1, 4, 5, 7])
    rp, rl = np.zeros(10, np.uint32), np.zeros(4, np.uint32)
    # remove primitive 1 (a light) of instance 0: primitive 5 (light 2) moves to 1
    edits.rearrange(insts, prims, aabbs, lights, cfg, [1], [0], rp, rl)
    assert insts["primitive_count"].tolist() == [5, 4]
    assert rp[1] == 0xFFFFFFFF and rp[5] == 1
    # light 0 removed; light 3 (last) moves into slot 0
    assert cfg["cube_light_count"][0] == 3 and cfg["light_count"][0] == 4
    assert rl.tolist() == [0xFFFFFFFF, 0, 0, 0]
    assert lights["instance_id"][:3].tolist() == [1, 0, 0]
    # light 2 followed its primitive from 5 to 1; light 3 (now 0) is inst 1 prim 1
    assert lights["primitive_id"][:3].tolist() == [1, 4, 1]
    assert prims["light_index"][6 + 1] == 0     # the moved light's primitive points at its new slot
    assert prims["light_index"][1] == 2         # the moved primitive keeps its light
    assert prims["light_index"][4] == 1


def test_rearrange_light_moves_from_the_tail():
    insts, prims, aabbs, lights, cfg = _scene([6], lights_at=[0, 2, 3, 5])
    rp, rl = np.zeros(6, np.uint32), np.zeros(4, np.uint32)
    edits.rearrange(insts, prims, aabbs, lights, cfg, [0, 2], [0], rp, rl)
    # primitives: n2 = 4, head marks [0, 2] take tail [4, 5]
    assert prims["material_index"][:4].tolist() == [4, 1, 5, 3]
    # lights 0, 1 removed; L2 = 2; tail kept lights [2, 3] -> slots [0, 1]
    assert rl.tolist() == [0xFFFFFFFF, 0xFFFFFFFF, 0, 1]
    assert lights["primitive_id"][:2].tolist() == [3, 2]   # light of prim 5 now at prim 2
    assert prims["light_index"][3] == 0 and prims["light_index"][2] == 1


def test_brush_window_and_instance_rule():
    W, H = 10, 8
    di = np.zeros(W * H, L.DI_INFO)
    di["distance"] = 1.0
    di["instance_id"] = 0
    di["primitive_id"] = np.arange(W * H)
    di["instance_id"][5 * W + 5] = 1          # another instance: skipped
    di["distance"][4 * W + 4] = 0.0                           # a miss: skipped
    insts = np.zeros(2, L.INSTANCE)
    insts["first_primitive_index"] = (0, 1000)
    prims, ins = edits.brush(di, W, H, (5, 4), 1, insts)
    want = sorted(y * W + x for y in (3, 4, 5) for x in (4, 5, 6) if (x, y) not in ((5, 5), (4, 4)))
    assert prims.tolist() == want and ins.tolist() == [0]
    # a window crossing the left edge selects nothing (unsigned lower corner)
    prims, ins = edits.brush(di, W, H, (0, 4), 1, insts)
    assert prims.size == 0
    # a missed centre selects nothing
    prims, ins = edits.brush(di, W, H, (4, 4), 1, insts)
    assert prims.size == 0


def test_oracle_frame_after_an_edit(oracle_lib):
    sc, W, H, cams, kw = build_case("grid16")
    r = oracle_lib.OracleRenderer(sc, W, H, **kw)
    for iv, ip in cams[:2]:
        r.render(iv, ip)
    n_before = int(r._keep[0]["primitive_count"].sum())
    prims, insts = r.erase((W // 2, H // 2), 3)
    assert prims.size > 0 and insts.tolist() == [0]
    assert int(r._keep[0]["primitive_count"].sum()) == n_before - prims.size
    remap_p = r._keep[7].copy()
    assert (remap_p[prims] == 0xFFFFFFFF).all()
    img = r.render(*cams[2])
    assert np.isfinite(img).all()
    assert r.prev_accel is None and not r._keep[7].any()
    r.close()
