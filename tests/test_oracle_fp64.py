"""The FP64 build of the oracle (the same shader code in double precision,
oracle/Makefile CT_ORACLE_FP64) and the error of the single-precision
results against it.  The CUDA path matches the FP32 oracle bit for bit on
these cases (test_gpu_parity), so these figures are its error too."""
import os
import sys

import numpy as np
import pytest

if __name__ == "__main__":
    _root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(_root, "cube-tracing_b200"), os.path.join(_root, "oracle"), os.path.dirname(__file__)]

from cases import CASES, PT_CASES, build_case  # noqa: E402

pyoracle = pytest.importorskip("pyoracle")
pytestmark = pytest.mark.skipif(not pyoracle.available(fp64=True), reason="FP64 oracle not built")

from cube_tracing import layouts as L  # noqa: E402


def test_fp64_layouts_match_the_library():
    i = pyoracle.info(fp64=True)
    w = pyoracle.widen
    assert (i.instance, i.aabb, i.primitive, i.material, i.light, i.light_config) == tuple(
        w(d).itemsize for d in (L.INSTANCE, L.AABB, L.PRIMITIVE, L.MATERIAL, L.LIGHT, L.LIGHT_CONFIG))
    assert (i.reservoir, i.di_info, i.velocity, i.path_reservoir) == tuple(
        w(d).itemsize for d in (L.RESERVOIR, L.DI_INFO, L.VELOCITY, L.PATH_RESERVOIR))
    assert (i.camera_view, i.status, i.world, i.restir) == tuple(
        w(d).itemsize for d in (L.CAMERA_VIEW, L.STATUS, L.WORLD, L.RESTIR))
    assert w(L.RESERVOIR).itemsize == 64 and w(L.DI_INFO).itemsize == 104


def test_fp64_build_is_double_precision():
    """One frame differs from the FP32 build in the low bits (and only there)."""
    sc, W, H, cams, kw = build_case("grid16")
    a = pyoracle.OracleRenderer(sc, W, H, **kw)
    b = pyoracle.OracleRenderer(sc, W, H, fp64=True, **kw)
    ia, ib = a.render(*cams[0]), b.render(*cams[0])
    assert ia.dtype == np.float32 and ib.dtype == np.float64
    assert not np.array_equal(ia.astype(np.float64), ib)
    assert np.allclose(ia, ib, rtol=1e-4, atol=1e-6)
    a.close()
    b.close()


@pytest.mark.parametrize("name", CASES + PT_CASES)
def test_fp32_error_against_fp64(name):
    """Every frame: ids, DI reservoir and PT path choices agree on at least
    99% of the hit pixels, and where both builds chose the same samples the
    image's relative error has a median below 1e-6 and a 99th percentile
    below 1e-3.  (Specular materials amplify it most: a metal's reflection
    or a dielectric's Fresnel choice turns on the last bits of a normal.)"""
    sc, W, H, cams, kw = build_case(name)
    a = pyoracle.OracleRenderer(sc, W, H, **kw)
    b = pyoracle.OracleRenderer(sc, W, H, fp64=True, **kw)
    for f, (iv, ip) in enumerate(cams):
        ia, ib = a.render(iv, ip), b.render(iv, ip)
        e = pyoracle.precision_error(a, b, ia, ib)
        assert e["ids_equal"] >= 0.99 and e["reservoirs_equal"] >= 0.99 and e["paths_equal"] >= 0.99, (name, f, e)
        assert e["image_rel_err"]["median"] < 1e-6 and e["image_rel_err"]["p99"] < 1e-3, (name, f, e)
    a.close()
    b.close()


def test_fp32_error_against_fp64_after_an_edit():
    """The same comparison on the frame after an erase (REMAP_BIT, the
    previous scene bound as tlas_previous): both builds remove the same
    voxels and choose the same samples."""
    sc, W, H, cams, kw = build_case("grid16_pt")
    a = pyoracle.OracleRenderer(sc, W, H, **kw)
    b = pyoracle.OracleRenderer(sc, W, H, fp64=True, **kw)
    for iv, ip in cams[:2]:
        a.render(iv, ip)
        b.render(iv, ip)
    ma, mb = a.erase((18, 14), 4), b.erase((18, 14), 4)
    assert ma[0].size > 0 and np.array_equal(ma[0], mb[0]) and np.array_equal(ma[1], mb[1])
    e = pyoracle.precision_error(a, b, a.render(*cams[2]), b.render(*cams[2]))
    assert e["ids_equal"] == 1.0 and e["reservoirs_equal"] >= 0.99 and e["paths_equal"] >= 0.99, e
    assert e["image_rel_err"]["median"] < 1e-6 and e["image_rel_err"]["p99"] < 1e-3, e
    a.close()
    b.close()


def table():
    """Markdown table of the last frame's error per case (python
    tests/test_oracle_fp64.py)."""
    rows = ["| case | ids | DI reservoirs | PT paths | median | p99 | max | p99 (all pixels) |",
            "|---|---|---|---|---|---|---|---|"]
    for name in CASES + PT_CASES:
        sc, W, H, cams, kw = build_case(name)
        a = pyoracle.OracleRenderer(sc, W, H, **kw)
        b = pyoracle.OracleRenderer(sc, W, H, fp64=True, **kw)
        for iv, ip in cams:
            ia, ib = a.render(iv, ip), b.render(iv, ip)
        e = pyoracle.precision_error(a, b, ia, ib)
        s, t = e["image_rel_err"], e["image_rel_err_all"]
        rows.append(f"| {name} | {e['ids_equal']:.4f} | {e['reservoirs_equal']:.4f} | {e['paths_equal']:.4f} | "
                    f"{s['median']:.1e} | {s['p99']:.1e} | {s['max']:.1e} | {t['p99']:.1e} |")
        a.close()
        b.close()
    return "\n".join(rows)


if __name__ == "__main__":
    print(table())
