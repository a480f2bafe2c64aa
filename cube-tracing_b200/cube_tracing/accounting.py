"""Algorithmic byte counts of the frame's kernels (the roofline numerator).

Bytes are counted from the reference's data layouts and pass structure, not
from this library's: a per-pixel record read or written by a pass counts its
reference struct size (DIRECT_ILLUMINATION_INFO 60 B, RESERVOIR 36 B,
VELOCITY 8 B, MATERIAL 84 B, LIGHT 40 B, RGBA32F texel 16 B), and every
ray counts 64 B (one 512-bit occupancy mask) per 8^3 brick it enters on its
way to the hit or to its end, plus the records a hit needs (AABB 24 B,
PRIMITIVE 8 B).  The per-launch counts (hit pixels, rays, bricks entered,
light candidates, neighbour and temporal records) come from the kernels'
work counters (CT_PARAM_COUNT_RAYS) in an untimed replay of the same frame;
they are properties of the frame, not of how the kernels run.
"""
DI, RES, VEL, MAT, LIGHT, TEXEL, AABB, PRIM, BRICK, PATH_RES, RGB = 60, 36, 8, 84, 40, 16, 24, 8, 64, 92, 12


def trace_bytes(c, pixels, taa):
    hits = c["hits"]
    misses = pixels - hits
    return (pixels * DI + hits * (VEL + AABB + PRIM) + misses * TEXEL * (2 if taa else 1) + c["brick_visits"] * BRICK)


def di_initial_bytes(c):
    hits = c["hits"]
    return (hits * (DI + VEL + MAT + RES + RES + 8) + c["temporal"] * (DI + MAT) + c["candidates"] * LIGHT +
            c["brick_visits"] * BRICK)


def di_shade_bytes(c, pixels, taa, final=True):
    hits = c["hits"]
    per_hit = DI + RES + MAT
    if final:
        per_hit += TEXEL * (2 if taa else 1) + RES + DI
    else:
        per_hit += RES
    misses = pixels - hits if final else 0
    return hits * per_hit + misses * 4 + c["neighbours"] * (DI + RES + MAT) + c["brick_visits"] * BRICK


def taa_bytes(hits_dispatched, pixels_dispatched):
    return pixels_dispatched * DI + hits_dispatched * (9 * DI + 9 * TEXEL + VEL + DI + TEXEL + TEXEL)


def pt_trace_bytes(c):
    """ReSTIR PT stage 0 (pass 1's indirect block): per hit pixel the DI
    record, material, velocity, the reprojected temporal path reservoir with
    its DI record and material, the written path reservoir, indirect colour
    and DI seed; per bounce hit the AABB, primitive and material records; per
    ray the bricks its walk enters."""
    hits = c["hits"]
    return (hits * (DI + MAT + VEL + PATH_RES + DI + MAT + PATH_RES + RGB + 4) +
            c["bounce_hits"] * (AABB + PRIM + MAT) + c["brick_visits"] * BRICK)


def pt_spatial_bytes(c, taa):
    """ReSTIR PT stage 1 (pass 2's indirect block and the final shading): per
    hit pixel its DI record, material, path reservoir, seed and image texel
    in, path reservoir, texel(s) and seed out; per valid neighbour its DI
    record, material and path reservoir plus the two reconnection vertices'
    AABB, primitive and material records; per ray the bricks entered."""
    hits = c["hits"]
    per_hit = DI + MAT + PATH_RES + 4 + TEXEL + PATH_RES + TEXEL * (2 if taa else 1) + 4
    return hits * per_hit + c["neighbours"] * (DI + MAT + PATH_RES + 2 * (AABB + PRIM + MAT)) + c["brick_visits"] * BRICK

