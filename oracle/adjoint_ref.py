"""CPU oracle of the adjoint renderer (ct_adjoint_forward / ct_adjoint_backward).

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the product package.

The renderer has no reference counterpart; what is pinned to the reference
is its path geometry: oracle_adjoint_paths (oracle_main.cpp) traces every
sample's vertices with the reference's own intersect(), compute_ray_origin
and random_cosine_direction in single precision, the precision of the CUDA
path, so both sides meet the same voxels.  On those vertices this module
restates the renderer's arithmetic:

  forward32  -- the image in float32 in the kernel's operation order (each
                sample: L += T * E[v], T *= a[v]; the samples summed in
                order, then times 1/spp), which the CUDA forward must match
                bit for bit;
  forward64  -- the same in float64;
  backward64 -- the gradient of a loss with image derivative d_image, in
                float64: d_emission[e(v_k)] += g T_k and
                d_albedo[v_k] += g T_k S_k with S_k the radiance gathered
                after v_k, g = d_image / spp.
"""
import ctypes

import numpy as np

import pyoracle

NONE = 0xFFFFFFFF


def paths(scene, inv_view, inv_proj, width, height, spp, depth, seed, rect, threads=0):
    """Vertices (global primitive indices) of every sample of every pixel of
    rect = (x0, y0, x1, y1): uint32 (rows * cols, spp, depth), NONE after a
    path's end."""
    lib = pyoracle.lib()
    lib.oracle_adjoint_paths.restype = ctypes.c_int
    lib.oracle_adjoint_paths.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    r = pyoracle.OracleRenderer(scene, width, height, threads=threads)
    try:
        pc = r.push_constant()
        x0, y0, x1, y1 = rect
        out = np.zeros(((y1 - y0) * (x1 - x0), spp, depth), np.uint32)
        iv = np.ascontiguousarray(inv_view, np.float32).reshape(16)
        ip = np.ascontiguousarray(inv_proj, np.float32).reshape(16)
        rc = np.array(rect, np.uint32)
        st = lib.oracle_adjoint_paths(ctypes.byref(pc), iv.ctypes.data, ip.ctypes.data, width, height, spp, depth,
                                      seed, rc.ctypes.data, out.ctypes.data, threads)
        if st != 0:
            raise ValueError("bad rect or depth")
    finally:
        r.close()
    return out


def _gather(verts, s, k, emitter_index):
    v = verts[:, s, k]
    valid = v != NONE
    vi = np.where(valid, v, 0).astype(np.int64)
    em = np.where(valid, emitter_index[vi], -1)
    return valid, vi, em


def forward32(verts, albedo, emission, emitter_index):
    """float32 image of the pixels (n, 3) in the CUDA kernel's order."""
    albedo = np.asarray(albedo, np.float32)
    emission = np.asarray(emission, np.float32)
    n, spp, depth = verts.shape
    sx = np.zeros((n, 3), np.float32)
    for s in range(spp):
        t = np.ones((n, 3), np.float32)
        lx = np.zeros((n, 3), np.float32)
        for k in range(depth):
            valid, vi, em = _gather(verts, s, k, emitter_index)
            emits = em >= 0
            lx[emits] = lx[emits] + t[emits] * emission[em[emits]]
            t[valid] = t[valid] * albedo[vi[valid]]
        sx = sx + lx
    inv = np.float32(1.0) / np.float32(spp)
    return sx * inv


def forward64(verts, albedo, emission, emitter_index):
    albedo = np.asarray(albedo, np.float64)
    emission = np.asarray(emission, np.float64)
    n, spp, depth = verts.shape
    acc = np.zeros((n, 3))
    for s in range(spp):
        t = np.ones((n, 3))
        for k in range(depth):
            valid, vi, em = _gather(verts, s, k, emitter_index)
            emits = em >= 0
            acc[emits] += t[emits] * emission[em[emits]]
            t[valid] *= albedo[vi[valid]]
    return acc / spp


def backward64(verts, albedo, emission, emitter_index, d_image):
    """(d_albedo, d_emission) in float64 for the pixels' d_image (n, 3)."""
    albedo = np.asarray(albedo, np.float64)
    emission = np.asarray(emission, np.float64)
    n, spp, depth = verts.shape
    g = np.asarray(d_image, np.float64) / spp
    ga = np.zeros(albedo.shape)
    ge = np.zeros(emission.shape)
    for s in range(spp):
        T = np.ones((depth, n, 3))
        t = np.ones((n, 3))
        gathered = [_gather(verts, s, k, emitter_index) for k in range(depth)]
        for k in range(depth):
            valid, vi, _ = gathered[k]
            T[k] = t
            t = np.where(valid[:, None], t * albedo[vi], t)
        S = np.zeros((n, 3))
        for k in range(depth - 1, -1, -1):
            valid, vi, em = gathered[k]
            gt = g * T[k]
            emits = em >= 0
            np.add.at(ge, em[emits], gt[emits])
            # the last vertex of a path gathers nothing after it (S = 0)
            np.add.at(ga, vi[valid], (gt * S)[valid])
            e = np.zeros((n, 3))
            e[emits] = emission[em[emits]]
            S = np.where(valid[:, None], albedo[vi] * S + e, 0.0)
    return ga, ge
