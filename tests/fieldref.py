"""CPU restatement of the walk's cell field (ct_accel_field): for every cell
of a grid and ray octant, the edge of the largest cube without occupied cells
that has the cell as its corner and extends in the octant's directions (the
part beyond the grid counts as empty), rounded down to the edges the 4-bit
codes stand for.  Test infrastructure: the library builds its field on the
GPU (k_field_step, k_field_grow, k_field_pack in csrc/ct_accel.cu)."""
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# the edges of the 16 field codes (CT_FIELD_EDGES0-3, csrc/ct_types.cuh)
FIELD_EDGES = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 15, 19, 24, 30)


def header_edges():
    """The code table as the CUDA header defines it."""
    src = open(os.path.join(ROOT, "cube-tracing_b200", "csrc", "ct_types.cuh")).read()
    words = [int(re.search(rf"#define CT_FIELD_EDGES{i} (0x[0-9A-Fa-f]+)u", src).group(1), 16) for i in range(4)]
    return tuple((w >> (8 * b)) & 255 for w in words for b in range(4))


def _flip(a, octant):
    if octant & 1:
        a = a[:, :, ::-1]
    if octant & 2:
        a = a[:, ::-1, :]
    if octant & 4:
        a = a[::-1, :, :]
    return a


def exact_edges(occ, octant, cap):
    """min(cap, largest empty forward cube edge) per cell; occ is [z, y, x]."""
    a = _flip(np.asarray(occ, bool), octant)
    Z, Y, X = a.shape
    k = np.where(a, 0, cap).astype(np.int32)
    # k(c) = 0 when occupied, else min(cap, 1 + min over the 7 forward
    # neighbours), a neighbour beyond the grid counting as cap; cap sweeps
    # reach the fixed point
    for _ in range(cap):
        p = np.pad(k, ((0, 1), (0, 1), (0, 1)), constant_values=cap)
        m = np.full_like(k, cap)
        for d in range(1, 8):
            dx, dy, dz = d & 1, (d >> 1) & 1, (d >> 2) & 1
            m = np.minimum(m, p[dz:dz + Z, dy:dy + Y, dx:dx + X])
        k = np.where(a, 0, np.minimum(cap, 1 + m)).astype(np.int32)
    return _flip(k, octant)


def coded_edges(occ, octant, edges=FIELD_EDGES):
    """exact_edges rounded down to the table's edges."""
    t = np.asarray(edges, np.int32)
    k = exact_edges(occ, octant, int(t[-1]))
    return t[np.searchsorted(t, k, side="right") - 1].astype(np.uint8)


def brute_edges(occ, octant, cap):
    """exact_edges by testing every cube directly (small grids only)."""
    a = _flip(np.asarray(occ, bool), octant)
    Z, Y, X = a.shape
    out = np.zeros(a.shape, np.int32)
    for z in range(Z):
        for y in range(Y):
            for x in range(X):
                e = 0
                while e < cap and not a[z:z + e + 1, y:y + e + 1, x:x + e + 1].any():
                    e += 1
                out[z, y, x] = e
    return _flip(out, octant)


def grid_occupancy(scene, instance, grid_min, shape):
    """[z, y, x] occupancy of an instance's grid: the voxels of its AABBs
    (integer voxel coordinates: AABB minimum / voxel edge)."""
    inst = scene.instances[instance]
    first, count = int(inst["first_primitive_index"]), int(inst["primitive_count"])
    mins = scene.aabbs["minimum"][first:first + count] / np.float32(scene.voxel_extent)
    v = np.floor(mins + 0.5).astype(np.int64) - np.asarray(grid_min, np.int64)
    occ = np.zeros(shape, bool)
    occ[v[:, 2], v[:, 1], v[:, 0]] = True
    return occ
