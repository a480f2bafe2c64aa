"""MagicaVoxel loading: the file format round trip and the reference loader's
layout of voxels, materials, lights and instances (map_loader.cpp:106-327)."""
import glob
import os

import numpy as np
import pytest

from cube_tracing import layouts as L
from cube_tracing import vox
from refdir import reference_dir

# the reference's shipped models, where its checkout is present
ASSETS = os.path.join(reference_dir(), "assets", "models")


def _palette():
    pal = np.zeros((256, 4), np.uint8)
    pal[:, 3] = 255
    pal[:, 0] = np.arange(256)
    pal[:, 1] = 255 - np.arange(256)
    pal[:, 2] = 7
    return pal


def test_write_read_round_trip():
    rng = np.random.default_rng(0)
    m0 = np.concatenate([rng.integers(0, 10, (50, 3)), rng.integers(1, 256, (50, 1))], axis=1).astype(np.uint8)
    m1 = np.array([[1, 2, 3, 4]], np.uint8)
    data = vox.write_vox([((10, 10, 10), m0), ((4, 5, 6), m1)], _palette(), emissive=(4, 17))
    models, pal, em = vox.read_vox(data)
    assert [m[0] for m in models] == [(10, 10, 10), (4, 5, 6)]
    assert np.array_equal(models[0][1], m0) and np.array_equal(models[1][1], m1)
    assert np.array_equal(pal, _palette())
    assert em == {4, 17}


def test_rejects_other_files():
    with pytest.raises(ValueError):
        vox.read_vox(b"RIFF" + bytes(16))


def test_layout_order_materials_and_lights():
    # model 0: three voxels given out of order, colour 3 twice, colour 5 emissive
    m0 = np.array([[1, 0, 1, 3], [0, 0, 0, 5], [0, 1, 0, 3]], np.uint8)
    # model 1 reuses colour 3: it gets its own material (per-model palette)
    m1 = np.array([[2, 2, 2, 3]], np.uint8)
    pal = _palette()
    sc = vox.scene_from_vox(*vox.read_vox(vox.write_vox([((2, 2, 2), m0), ((3, 3, 3), m1)], pal, (5,))),
                            voxel_extent=0.5, axis="Z_BOTTOM_TOP")
    # z, y, x order (x fastest): (0,0,0) (0,1,0) (1,0,1), then model 1
    assert np.array_equal(sc.aabbs["minimum"], np.array([[0, 0, 0], [0, 0.5, 0], [0.5, 0, 0.5], [1, 1, 1]],
                                                          np.float32))
    assert np.array_equal(sc.aabbs["maximum"] - sc.aabbs["minimum"], np.full((4, 3), 0.5, np.float32))
    assert list(sc.primitives["material_index"]) == [0, 1, 1, 2]
    assert list(sc.primitives["light_index"]) == [0, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF]
    assert sc.materials.shape[0] == 3
    assert np.allclose(sc.materials["diffuse"][0], pal[4, :3] / np.float32(255.0))
    assert np.array_equal(sc.materials["emission"][0], pal[4, :3].astype(np.float32) / np.float32(255.0))
    assert not sc.materials["emission"][1:].any()
    assert (sc.materials["type"] == 0).all() and (sc.materials["illum"] == 3).all()
    assert (sc.materials[["shininess", "roughness", "ior", "dissolve"]].tolist() == [(1.0,) * 4] * 3)
    lt = sc.cube_lights
    assert lt.shape[0] == 1 and lt["type"][0] == L.LIGHT_CUBE
    assert np.array_equal(lt["position"][0], np.float32([0.25, 0.25, 0.25]))
    assert (lt["instance_id"][0], lt["primitive_id"][0], lt["size"][0]) == (0, 0, 0.5)
    assert list(sc.instances["first_primitive_index"]) == [0, 3]
    assert list(sc.instances["primitive_count"]) == [3, 1]
    assert np.array_equal(sc.instances["transform"], np.tile(np.eye(4, dtype=np.float32).ravel(), (2, 1)))
    cfg = sc.light_config[0]
    assert (cfg["cube_light_count"], cfg["light_count"], cfg["cube_light_pdf"]) == (1, 1, 1.0)


@pytest.mark.parametrize("axis,perm", [("Z_BOTTOM_TOP", (0, 1, 2)), ("X_BOTTOM_TOP", (1, 2, 0)),
                                       ("Y_TOP_BOTTOM", (2, 0, 1))])
def test_axis_direction(axis, perm):
    m = np.array([[1, 2, 3, 1]], np.uint8)
    sc = vox.scene_from_vox([((4, 4, 4), m)], _palette(), set(), axis=axis)
    s = (1, 2, 3)
    assert tuple(sc.aabbs["minimum"][0]) == tuple(float(s[p]) for p in perm)


def test_duplicate_voxel_keeps_the_last():
    m = np.array([[1, 1, 1, 2], [1, 1, 1, 9]], np.uint8)
    sc = vox.scene_from_vox([((2, 2, 2), m)], _palette(), set())
    assert sc.voxel_count == 1
    assert np.allclose(sc.materials["diffuse"][0], _palette()[8, :3] / 255.0)


@pytest.mark.skipif(not os.path.isdir(ASSETS), reason="reference assets not present")
def test_reference_assets_parse():
    files = sorted(glob.glob(os.path.join(ASSETS, "*.vox")))
    assert files
    for f in files:
        models, pal, em = vox.read_vox(f)
        assert models
        for size, v in models:
            assert (v[:, :3] < np.array(size)).all() and (v[:, 3] > 0).all()
        sc = vox.load_vox(f)
        assert sc.voxel_count == sum(len(np.unique(v[:, :3], axis=0)) for _, v in models)
        assert sc.primitives["material_index"].max() < sc.materials.shape[0]
        if os.path.basename(f) == "room.vox":
            assert em and sc.cube_lights.shape[0] > 0
