"""Traversal parity: the library's voxel walk (ct_trace_visibility,
ct_trace_closest) against the reference's own is_vertex_visible and
traceRayEXT + intersection shader (the oracle), ray by ray, bit for bit.
Includes rays along voxel faces, edges and corners, where the box test's
rounding decides which voxel is hit."""
import ctypes
import zlib

import numpy as np
import pytest

import rays
from cases import build_case
from cube_tracing import layouts as L
from cube_tracing import native


def gpu_queries(accel, records, closest):
    import torch
    q = torch.from_numpy(records.view(np.uint8).copy()).cuda()
    n = records.shape[0]
    out = torch.zeros(n * (16 if closest else 1), dtype=torch.uint8, device="cuda")
    fn = native.lib().ct_trace_closest if closest else native.lib().ct_trace_visibility
    native.check("ct_trace_*", fn(accel.handle, q.data_ptr(), n, out.data_ptr(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return o.view(L.RAY_HIT) if closest else o


SETS = {
    "shadow": (rays.shadow_rays, False),
    "segments": (rays.random_segments, False),
    "degenerate_vis": (rays.degenerate_rays, False),
    "camera": (rays.camera_rays, True),
    "degenerate_closest": (rays.degenerate_rays, True),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["grid16", "terrain32", "grid32_allfeatures", "instances16"])
@pytest.mark.parametrize("kind", list(SETS))
def test_queries_match_reference(oracle_lib, case, kind):
    from cube_tracing.frame import SceneBuffers
    sc, W, H, cams, kw = build_case(case)
    gen, closest = SETS[kind]
    recs = gen(sc, 20000, seed=zlib.crc32(f"{case}/{kind}".encode()))
    ora = oracle_lib.OracleRenderer(sc, 8, 8)
    ref = ora.queries(recs, closest=closest)
    sb = SceneBuffers(sc)
    got = gpu_queries(sb.accel, recs, closest)
    if closest:
        ok = (got["instance_id"] == ref["instance_id"]) & (got["primitive_id"] == ref["primitive_id"]) & \
             (got["t"].view(np.uint32) == ref["t"].view(np.uint32))
    else:
        ok = got == ref
    bad = np.nonzero(~ok)[0]
    msg = [f"{len(bad)} of {len(recs)} rays differ"] + [
        f"ray {i}: o={recs[i]['origin'].tolist()} d={recs[i]['direction'].tolist()} dist={recs[i]['distance']} "
        f"flags={recs[i]['flags']} target={recs[i]['target_primitive']} gpu={got[i]} ref={ref[i]}" for i in bad[:5]]
    assert len(bad) == 0, "\n".join(msg)
    if not closest:
        assert 0 < ref.mean() < 1  # both outcomes occur


@pytest.mark.gpu
def test_closest_tie_across_bricks(oracle_lib):
    """A camera ray that leaves the voxel it starts in through the face it
    shares with the voxel below, in the next brick: both are hit at the same
    distance and the lower primitive index wins.  The walk's stop test must
    still enter the next brick although the grid-local exit distance, with
    a direction component of 0.087, rounds above the hit distance."""
    from cube_tracing.frame import SceneBuffers
    sc, W, H, cams, kw = build_case("grid16")
    r = np.zeros(1, L.RAY_QUERY)
    r["origin"] = (0.36978381872177124, 15.068591117858887, 0.007090447004884481)
    r["direction"] = (0.6260949969291687, -0.08651454001665115, 0.7749324440956116)
    r["distance"] = 1e9
    ref = oracle_lib.OracleRenderer(sc, 8, 8).queries(r, closest=True)
    got = gpu_queries(SceneBuffers(sc).accel, r, True)
    assert int(ref["primitive_id"][0]) == 69
    assert got.tobytes() == ref.tobytes()
