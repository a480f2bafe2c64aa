"""CPU restatement of cube-tracing's scene edits: the voxel brush and the
primitive rearrangement.

TEST INFRASTRUCTURE ONLY: the checker of ct_brush / ct_rearrange, imported
by tests/ and never by the product package.

The reference runs these as Slang compute shaders (no C++ compilation of
them is possible here), so they are restated in numpy:

  brush      entry_brush + delete_primitive_from_instance
             (src/shaders/slang/compute/squared_brush.slang:37-133)
  rearrange  entry_rearragement (src/shaders/slang/compute/rearrangement.slang:56-204)
             with the bookkeeping ACCEL_STRUCT_MNGR does around it
             (accel_struct_mngr.cpp:607-816 cube lights and remap entries,
             2679-2800 bitmask readback and reset).

The reference's rearrangement pairs marked primitives with replacements per
GPU thread and leaves the pairing order to its scan; the rule restated here
(and built by the CUDA path) is the deterministic one its comments describe:
per instance of n primitives with k marked, the j-th marked primitive below
n - k takes the j-th unmarked primitive at or above n - k.  With one marked
primitive this is the reference's CPU path, swap with the last
(delete_aabb_device_buffer, accel_struct_mngr.cpp:607-731), and cube lights
follow the same rule over the light list (update_light_remapping_buffer,
:775-816).
"""
import numpy as np

U32 = 0xFFFFFFFF


def brush(prev_di, width, height, pixel, window, instances):
    """entry_brush over every pixel.  Returns (marked global primitive
    indices, marked instance ids), both sorted; the brush counter holds their
    lengths."""
    cx, cy = int(pixel[0]), int(pixel[1])
    empty = (np.zeros(0, np.int64), np.zeros(0, np.int64))
    if cx >= width or cy >= height:
        return empty
    centre = prev_di[cy * width + cx]
    if not centre["distance"] > 0.0:
        return empty
    # uint2(pixel - window): a wrapped lower corner stays huge
    min_x, min_y = (cx - window) & U32, (cy - window) & U32
    max_x = min((cx + window) & U32, width - 1 if width else 0)
    max_y = min((cy + window) & U32, height - 1 if height else 0)
    ys, xs = np.mgrid[0:height, 0:width]
    xs, ys = xs.ravel(), ys.ravel()
    inside = (xs >= min_x) & (xs <= max_x) & (ys >= min_y) & (ys <= max_y)
    d = prev_di[ys * width + xs]
    sel = inside & (d["distance"] > 0.0) & (d["instance_id"] == centre["instance_id"])
    inst = d["instance_id"][sel].astype(np.int64)
    prim = instances["first_primitive_index"][inst].astype(np.int64) + d["primitive_id"][sel]
    return np.unique(prim), np.unique(inst)


def _moved_primitive(instances, remap_p, inst_id, prim_id):
    # ids outside the primitive table (the .vox loader's cube lights carry a
    # global index, map_loader.cpp:285) are left as they are
    if inst_id >= instances.shape[0]:
        return prim_id
    if prim_id < instances["primitive_count"][inst_id]:
        return prim_id
    g = int(instances["first_primitive_index"][inst_id]) + prim_id
    return int(remap_p[g]) if g < remap_p.shape[0] else prim_id


def rearrange(instances, primitives, aabbs, cube_lights, light_config, marked_prims, marked_insts, remap_p, remap_l):
    """Removes the marked primitives in place.  remap_p / remap_l (uint32)
    must be zero on entry; they receive 0xFFFFFFFF at removed entries and the
    new index at moved ones."""
    marked = np.zeros(primitives.shape[0], bool)
    marked[np.asarray(marked_prims, np.int64)] = True
    for i in sorted(int(v) for v in marked_insts):
        f = int(instances["first_primitive_index"][i])
        n = int(instances["primitive_count"][i])
        m = marked[f:f + n]
        k = int(m.sum())
        if k == 0:
            continue
        n2 = n - k
        dst = f + np.nonzero(m[:n2])[0]
        src = f + n2 + np.nonzero(~m[n2:])[0]
        assert dst.shape == src.shape
        primitives[dst] = primitives[src]
        aabbs[dst] = aabbs[src]
        remap_p[src] = (dst - f).astype(np.uint32)
        remap_p[f + np.nonzero(m)[0]] = U32
        instances["primitive_count"][i] = n2
    cfg = light_config[0]
    L = int(cfg["cube_light_count"])
    if L == 0:
        return
    removed = np.zeros(L, bool)
    for x in range(L):
        ii, pp = int(cube_lights["instance_id"][x]), int(cube_lights["primitive_id"][x])
        if ii < instances.shape[0]:
            g = int(instances["first_primitive_index"][ii]) + pp
            removed[x] = g < marked.shape[0] and marked[g]
    remap_l[:L] = np.where(removed, U32, 0).astype(np.uint32)
    m = int(removed.sum())
    L2 = L - m
    for x in range(L2 if m else L):
        if not removed[x]:
            cube_lights["primitive_id"][x] = _moved_primitive(instances, remap_p, int(cube_lights["instance_id"][x]),
                                                              int(cube_lights["primitive_id"][x]))
    if m == 0:
        return
    dst = np.nonzero(removed[:L2])[0]
    src = L2 + np.nonzero(~removed[L2:])[0]
    assert dst.shape == src.shape
    for s, d in zip(src.tolist(), dst.tolist()):
        lt = cube_lights[s].copy()
        ii = int(lt["instance_id"])
        lt["primitive_id"] = _moved_primitive(instances, remap_p, ii, int(lt["primitive_id"]))
        cube_lights[d] = lt
        remap_l[s] = d
        if ii < instances.shape[0]:
            g = int(instances["first_primitive_index"][ii]) + int(lt["primitive_id"])
            if g < primitives.shape[0]:
                primitives["light_index"][g] = d
    cfg["cube_light_count"] = L2
    cfg["light_count"] = max(int(cfg["light_count"]) - m, 0)
