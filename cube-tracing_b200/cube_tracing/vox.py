"""MagicaVoxel (.vox) scenes, laid out the way cube-tracing's loader does it
(src/gvox/map_loader.cpp:47-338).

The reference reads .vox files through gvox's MagicaVoxel adapter (gvox is
not vendored; its version is not pinned in the repository).  This module
reads the published MagicaVoxel file format itself (a RIFF-like chunk tree:
"VOX " version, MAIN with SIZE/XYZI model pairs, RGBA palette, and the MATL
or older MATT material chunks) and applies the reference's mapping per model:

  * voxels in z, y, x order (x fastest) over the model extent
    (map_loader.cpp:106-110), one AABB per voxel with minimum
    grid * VOXEL_EXTENT and maximum (grid + 1) * VOXEL_EXTENT, the grid
    coordinate permuted by the loader's axis direction (:228-263);
  * one Lambertian material per distinct palette index within a model
    (:183-222): diffuse = rgb / 255, emission = emissive rgb / 255 (flux is
    not implemented by the reference, so it is 1), shininess, roughness, ior
    and dissolve 1, illum 3;
  * one cube light per emissive voxel (:275-296): position the voxel centre,
    emissive the material's emission, instance_info (instance, global
    primitive index), size VOXEL_EXTENT; PRIMITIVE.light_index points at it,
    other voxels carry 0xFFFFFFFF;
  * one instance per model with the identity transform (:319-327).

A palette entry is emissive when its material is MagicaVoxel's emit material
(MATL `_type` = `_emit`, or MATT type 3); its emissivity colour is the
palette colour.
"""
import os
import struct

import numpy as np

from . import layouts as L
from .scenes import Scene

# permutation of the sample position into the grid (x_grid, y_grid, z_grid)
AXIS = {
    "Z_BOTTOM_TOP": (0, 1, 2), "Z_TOP_BOTTOM": (0, 1, 2),
    "X_BOTTOM_TOP": (1, 2, 0), "X_TOP_BOTTOM": (1, 2, 0),
    "Y_BOTTOM_TOP": (2, 0, 1), "Y_TOP_BOTTOM": (2, 0, 1),
}


def _default_palette():
    # MagicaVoxel's default palette is 256 fixed colours; files written by the
    # editor always carry RGBA.  Without one, a grey ramp stands in.
    p = np.zeros((256, 4), np.uint8)
    p[:, 0] = p[:, 1] = p[:, 2] = np.arange(256, dtype=np.uint8)
    p[:, 3] = 255
    return p


def _read_dict(b, i):
    n, = struct.unpack_from("<i", b, i)
    i += 4
    d = {}
    for _ in range(n):
        kl, = struct.unpack_from("<i", b, i)
        k = b[i + 4:i + 4 + kl].decode("latin-1")
        i += 4 + kl
        vl, = struct.unpack_from("<i", b, i)
        v = b[i + 4:i + 4 + vl].decode("latin-1")
        i += 4 + vl
        d[k] = v
    return d, i


def read_vox(data):
    """Parses .vox bytes (or a path).  Returns (models, palette, emissive)
    with models a list of (size (sx, sy, sz), voxels (n, 4) uint8 x y z
    colour index), palette (256, 4) uint8 where entry i is colour index i + 1,
    and emissive a set of colour indices."""
    if not isinstance(data, (bytes, bytearray, memoryview)):
        with open(data, "rb") as f:
            data = f.read()
    b = bytes(data)
    if b[:4] != b"VOX ":
        raise ValueError("not a MagicaVoxel file")
    i = 8
    if b[i:i + 4] != b"MAIN":
        raise ValueError("MAIN chunk missing")
    n, m = struct.unpack_from("<ii", b, i + 4)
    i += 12 + n
    end = i + m
    models, size, palette, emissive = [], None, None, set()
    while i < end:
        cid = b[i:i + 4]
        n, m = struct.unpack_from("<ii", b, i + 4)
        body = i + 12
        if cid == b"SIZE":
            size = struct.unpack_from("<iii", b, body)
        elif cid == b"XYZI":
            cnt, = struct.unpack_from("<i", b, body)
            vox = np.frombuffer(b, np.uint8, count=4 * cnt, offset=body + 4).reshape(cnt, 4).copy()
            if size is None:
                raise ValueError("XYZI before SIZE")
            models.append((size, vox))
        elif cid == b"RGBA":
            palette = np.frombuffer(b, np.uint8, count=1024, offset=body).reshape(256, 4).copy()
        elif cid == b"MATL":
            mid, = struct.unpack_from("<i", b, body)
            props, _ = _read_dict(b, body + 4)
            if props.get("_type") == "_emit" and 1 <= mid <= 255:
                emissive.add(mid)
        elif cid == b"MATT":
            mid, mtype = struct.unpack_from("<ii", b, body)
            if mtype == 3 and 1 <= mid <= 255:
                emissive.add(mid)
        i = body + n + m
    if palette is None:
        palette = _default_palette()
    return models, palette, emissive


def scene_from_vox(models, palette, emissive, voxel_extent=1.0, axis="Z_BOTTOM_TOP", name="vox"):
    """The reference loader's layout of the parsed models (see the module
    docstring)."""
    e = np.float32(voxel_extent)
    perm = AXIS[axis]
    aabbs, prims, mats, lights, insts = [], [], [], [], []
    n_prim = 0
    for inst_index, (size, vox) in enumerate(models):
        sx, sy, sz = size
        # z, y, x order over the extent (x fastest); a later voxel at the same
        # position replaces an earlier one, as a dense sample would
        key = (vox[:, 2].astype(np.int64) * sy + vox[:, 1]) * sx + vox[:, 0]
        order = np.argsort(key, kind="stable")
        key, vox = key[order], vox[order]
        last = np.ones(key.shape[0], bool)
        last[:-1] = key[1:] != key[:-1]
        key, vox = key[last], vox[last]
        palette_index = {}
        first = n_prim
        for (x, y, z, c) in vox:
            rgb = palette[c - 1, :3].astype(np.float32) if c > 0 else np.zeros(3, np.float32)
            light = c in emissive and bool(np.any(palette[c - 1, :3] != 0))
            emission = (rgb / np.float32(255.0)) * np.float32(1.0) if light else np.zeros(3, np.float32)
            if c not in palette_index:
                palette_index[c] = len(mats)
                m = np.zeros(1, L.MATERIAL)[0]
                m["type"] = 0
                m["diffuse"] = rgb / np.float32(255.0)
                m["emission"] = emission
                m["shininess"] = 1.0
                m["roughness"] = 1.0
                m["ior"] = 1.0
                m["dissolve"] = 1.0
                m["illum"] = 3
                mats.append(m)
            s = (int(x), int(y), int(z))
            g = np.array([s[perm[0]], s[perm[1]], s[perm[2]]], np.float32)
            a = np.zeros(1, L.AABB)[0]
            a["minimum"] = g * e
            a["maximum"] = (g + np.float32(1.0)) * e
            aabbs.append(a)
            p = np.zeros(1, L.PRIMITIVE)[0]
            p["material_index"] = palette_index[c]
            p["light_index"] = 0xFFFFFFFF
            if light:
                lt = np.zeros(1, L.LIGHT)[0]
                lt["position"] = g * e + e * np.float32(0.5)
                lt["emissive"] = emission
                lt["instance_id"] = inst_index
                lt["primitive_id"] = n_prim
                lt["size"] = e
                lt["type"] = L.LIGHT_CUBE
                p["light_index"] = len(lights)
                lights.append(lt)
            prims.append(p)
            n_prim += 1
        inst = np.zeros(1, L.INSTANCE)[0]
        inst["transform"] = np.eye(4, dtype=np.float32).reshape(-1, order="F")
        inst["first_primitive_index"] = first
        inst["primitive_count"] = n_prim - first
        insts.append(inst)
    as_arr = lambda rows, dt: np.array(rows, dt) if rows else np.zeros(0, dt)
    lights_a = as_arr(lights, L.LIGHT)
    cfg = np.zeros(1, L.LIGHT_CONFIG)
    cfg["cube_light_count"] = lights_a.shape[0]
    cfg["cube_light_pdf"] = 1.0 / max(lights_a.shape[0], 1)
    cfg["light_count"] = lights_a.shape[0]
    aabbs_a = as_arr(aabbs, L.AABB)
    if aabbs_a.shape[0]:
        edge = tuple(int(v) for v in np.ceil(aabbs_a["maximum"].max(axis=0) / e))
    else:
        edge = (0, 0, 0)
    return Scene(as_arr(insts, L.INSTANCE), aabbs_a, as_arr(prims, L.PRIMITIVE),
                 as_arr(mats, L.MATERIAL), lights_a, np.zeros(0, L.LIGHT), np.zeros(0, L.LIGHT), cfg,
                 float(voxel_extent), edge, name, {"models": len(models)})


def load_vox(path, voxel_extent=1.0, axis="X_BOTTOM_TOP"):
    """Reads a .vox file into a Scene.  The reference loads its maps and
    models with the X_BOTTOM_TOP axis direction (main.cpp:1046-1103)."""
    models, palette, emissive = read_vox(path)
    return scene_from_vox(models, palette, emissive, voxel_extent, axis, os.path.basename(str(path)))


def write_vox(models, palette=None, emissive=()):
    """A minimal .vox file (SIZE/XYZI per model, RGBA, one MATL per emissive
    palette index): for tests and for exporting synthetic scenes."""
    def chunk(cid, content, children=b""):
        return cid + struct.pack("<ii", len(content), len(children)) + content + children
    kids = b""
    for size, vox in models:
        vox = np.ascontiguousarray(vox, np.uint8)
        kids += chunk(b"SIZE", struct.pack("<iii", *size))
        kids += chunk(b"XYZI", struct.pack("<i", vox.shape[0]) + vox.tobytes())
    if palette is not None:
        kids += chunk(b"RGBA", np.ascontiguousarray(palette, np.uint8).tobytes())
    for mid in sorted(emissive):
        props = {"_type": "_emit", "_emit": "1.0"}
        body = struct.pack("<ii", mid, len(props))
        for k, v in props.items():
            body += struct.pack("<i", len(k)) + k.encode() + struct.pack("<i", len(v)) + v.encode()
        kids += chunk(b"MATL", body)
    return b"VOX " + struct.pack("<i", 150) + chunk(b"MAIN", b"", kids)
