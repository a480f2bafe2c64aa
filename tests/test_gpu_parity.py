"""Parity of the CUDA path (libct.so through the C ABI) with the CPU oracle
(the reference's shaders compiled as C++) on the same seeded workloads.

Bar (per pixel, every frame):
  * bit-exact: hit/miss, first-hit (instance, primitive) ids, material index,
    DI seed and confidence; reservoir light index Y, light type, light seed
    and sample count M;
  * bit-exact is also expected for positions, normals, distances, velocities
    and the reservoirs' float fields, and checked within RTOL otherwise;
  * radiance (output image, reservoir F, W_y, W_sum) within RTOL = 1e-4
    relative (FP32), plus an absolute floor of 1e-6.
"""
import os

import numpy as np
import pytest

from cases import CASES, PT_CASES, build_case, frame_keys
from cube_tracing import layouts as L

RTOL = 1e-4
ATOL = 1e-6
HERE = os.path.dirname(os.path.abspath(__file__))


def close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    return both_nan | (np.abs(a - b) <= RTOL * np.maximum(np.abs(a), np.abs(b)) + ATOL)


def where(mask, W):
    idx = np.nonzero(~mask)[0][:5]
    return [(int(i % W), int(i // W)) for i in idx]


def compare_frame(tag, W, gpu, ref):
    """gpu/ref: dict key -> structured arrays (FRAME_KEYS) + 'image'."""
    problems = []
    dg, do = gpu["di"], ref["di"]
    hit = do["distance"] > 0
    if not np.array_equal(dg["distance"] > 0, hit):
        problems.append(f"{tag} hit mask differs at {where((dg['distance'] > 0) == hit, W)}")
    for f in ("seed",):
        m = dg[f] == do[f]
        if not m.all():
            problems.append(f"{tag} di.{f} differs at {int((~m).sum())} px {where(m, W)}")
    for f in ("instance_id", "primitive_id", "mat_index", "confidence"):
        m = (dg[f] == do[f]) | ~hit
        if not m.all():
            problems.append(f"{tag} di.{f} differs at {int((~m).sum())} px {where(m, W)}")
    for f in ("position", "normal", "distance", "ray_origin"):
        a, b = dg[f], do[f]
        m = close(a, b)
        m = m.reshape(m.shape[0], -1).all(axis=1) | ~hit
        if not m.all():
            problems.append(f"{tag} di.{f} off at {int((~m).sum())} px {where(m, W)}")
    vg, vo = gpu["velocity"]["velocity"], ref["velocity"]["velocity"]
    m = close(vg, vo).all(axis=1) | ~hit
    if not m.all():
        problems.append(f"{tag} velocity off at {int((~m).sum())} px {where(m, W)}")
    for key in ("intermediate_reservoir", "previous_reservoir"):
        rg, ro = gpu[key], ref[key]
        for f in ("Y", "l_type", "seed", "M"):
            m = (rg[f] == ro[f]) | ~hit
            if not m.all():
                problems.append(f"{tag} {key}.{f} differs at {int((~m).sum())} px {where(m, W)}")
        for f in ("W_y", "W_sum", "F"):
            m = close(rg[f], ro[f])
            m = m.reshape(m.shape[0], -1).all(axis=1) | ~hit
            if not m.all():
                problems.append(f"{tag} {key}.{f} off at {int((~m).sum())} px {where(m, W)}")
    for key in ("output_path_reservoir", "temporal_path_reservoir"):
        if key not in ref:
            continue
        rg, ro = gpu[key], ref[key]
        for f in ("path_flags", "rc_random_seed", "init_random_seed", "rc_instance_id", "rc_primitive_id", "M"):
            m = (rg[f] == ro[f]) | ~hit
            if not m.all():
                problems.append(f"{tag} {key}.{f} differs at {int((~m).sum())} px {where(m, W)}")
        for f in ("weight", "F", "light_pdf", "cached_jacobian", "rc_hit", "rc_vertex_wi", "rc_vertex_irradiance"):
            m = close(rg[f], ro[f])
            m = m.reshape(m.shape[0], -1).all(axis=1) | ~hit
            if not m.all():
                problems.append(f"{tag} {key}.{f} off at {int((~m).sum())} px {where(m, W)}")
    if "indirect_color" in ref:
        m = close(gpu["indirect_color"], ref["indirect_color"]).reshape(-1, 3).all(axis=1)
        if not m.all():
            problems.append(f"{tag} indirect_color off at {int((~m).sum())} px {where(m, W)}")
    ig, io = gpu["image"].reshape(-1, 4), ref["image"].reshape(-1, 4)
    m = close(ig, io).all(axis=1)
    if not m.all():
        problems.append(f"{tag} image off at {int((~m).sum())} px {where(m, W)} "
                        f"max rel {np.max(np.abs(ig - io) / (np.abs(io) + 1e-6)):.3g}")
    return problems


def gpu_frame(r, img, keys):
    import torch
    torch.cuda.synchronize()
    out = {k: r.read(k) for k in keys}
    out["image"] = img.cpu().numpy()
    return out


def ref_frame(r, img, keys):
    out = {k: r.buf[k].copy() for k in keys}
    out["image"] = img.copy()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES + PT_CASES)
def test_gpu_matches_oracle(oracle_lib, name):
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    problems = []
    for f, (iv, ip) in enumerate(cams):
        ro = ref_frame(ora, ora.render(iv, ip), frame_keys(name))
        rg = gpu_frame(gpu, gpu.render(iv, ip), frame_keys(name))
        assert gpu.device_error() == (0, 0, 0)
        problems += compare_frame(f"{name} frame {f}", W, rg, ro)
    assert not problems, "\n".join(problems)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES + PT_CASES)
def test_gpu_matches_golden_fixture(name):
    """Same comparison against the committed fixture (no oracle library)."""
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    gpu = Renderer(sc, W, H, **kw)
    problems = []
    for f, (iv, ip) in enumerate(cams):
        rg = gpu_frame(gpu, gpu.render(iv, ip), frame_keys(name))
        ro = {k: L.view_buffer(k, g[f"f{f}_{k}"]) for k in frame_keys(name)}
        ro["image"] = g[f"f{f}_image"]
        problems += compare_frame(f"{name} frame {f}", W, rg, ro)
    assert not problems, "\n".join(problems)


@pytest.mark.gpu
def test_deep_paths_reach_the_last_rounds():
    """room16_deep_pt (max depth 12 in a closed room) runs paths past the 8
    wavefront rounds, so its parity cases above cover the kernel that
    finishes the longer paths: the same frame traces more bounce rays than
    at max depth 8, where no path goes past 8 bounces."""
    import torch
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case("room16_deep_pt")
    counts = {}
    for depth in (8, 12):
        r = Renderer(sc, W, H, count_rays=True, **dict(kw, max_depth=depth))
        r.render(*cams[0])
        torch.cuda.synchronize()
        counts[depth] = r.ray_counts()["bounce"]
        assert r.device_error() == (0, 0, 0)
    assert counts[12] > counts[8], counts


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["grid16_materials_brdf_pt", "glass_inside_brdf_pt", "grid32_allfeatures_pt"])
@pytest.mark.parametrize("byte", [0x02, 0xFF])
def test_stale_workspace_does_not_leak(oracle_lib, name, byte):
    """The frame's scratch (queues, answer slots, stored re-evaluations) is
    written before it is read: the renderer's workspace filled with a byte
    pattern before every frame (0x02 is the RIS visibility pass's skip
    marker, 0xFF makes every float NaN) still gives the oracle's frames."""
    from cube_tracing.frame import Renderer
    sc, W, H, cams, kw = build_case(name)
    ora = oracle_lib.OracleRenderer(sc, W, H, **kw)
    gpu = Renderer(sc, W, H, **kw)
    problems = []
    for f, (iv, ip) in enumerate(cams):
        gpu.workspace.fill_(byte)
        ro = ref_frame(ora, ora.render(iv, ip), frame_keys(name))
        rg = gpu_frame(gpu, gpu.render(iv, ip), frame_keys(name))
        assert gpu.device_error() == (0, 0, 0)
        problems += compare_frame(f"{name} frame {f}", W, rg, ro)
    assert not problems, "\n".join(problems)
    ora.close()
