"""Path-replay adjoint over per-voxel albedo and emission, through the C ABI
(ct_adjoint_forward / ct_adjoint_backward, include/ct.h).

The reference's renderer is not differentiable; this is the plain
Lambertian path tracer of its ReSTIR PT stage (closest hits of
intersect(), cosine-weighted bounces, bounce.glsl:9-125,
rcall_scatter.glsl:74-86) reduced to what an inverse-rendering loop needs:
the image as a function of per-voxel albedo and per-emitter radiance, and
the gradient of an image loss with respect to both, computed by replaying
every path from its RNG counters instead of storing it.

  AdjointScene     -- the differentiable-rendering workload: a seeded voxel
                      grid, its emitters, hidden target parameters, camera
  AdjointRenderer  -- forward (image) and backward (gradients) on the device
"""
from dataclasses import dataclass
import ctypes

import numpy as np
import torch

from . import layouts as L
from . import native
from . import scenes
from .frame import Accel, _dev


@dataclass
class AdjointScene:
    scene: scenes.Scene
    emitter_index: np.ndarray   # int32 per primitive: row of the emission table or -1
    albedo_target: np.ndarray   # float32 (n_prim, 3), hidden
    emission_target: np.ndarray  # float32 (n_emit, 3), hidden
    albedo_init: np.ndarray     # float32 (n_prim, 3)
    emission_init: np.ndarray   # float32 (n_emit, 3)
    inv_view: np.ndarray
    inv_proj: np.ndarray
    width: int
    height: int


def scene_tables(sc, inv_view, inv_proj, width, height):
    """An AdjointScene whose parameters are a loaded scene's own: per-voxel
    albedo from its materials' diffuse colour, emitters and their radiance
    from its cube lights' materials (the "target" and "init" are the same)."""
    n = sc.aabbs.shape[0]
    mats = sc.materials
    mi = sc.primitives["material_index"].astype(np.int64)
    albedo = np.ascontiguousarray(mats["diffuse"][mi], np.float32)
    emit = np.full(n, -1, np.int32)
    light_prims = sc.cube_lights["primitive_id"].astype(np.int64)
    emit[light_prims] = np.arange(light_prims.shape[0], dtype=np.int32)
    emission = np.ascontiguousarray(mats["emission"][mi[light_prims]], np.float32)
    return AdjointScene(sc, emit, albedo, emission, albedo, emission, inv_view, inv_proj, width, height)


def adjoint_scene(edge=128, occupancy=0.25, emissive_fraction=0.01, seed=3, target_seed=4, width=512, height=512,
                  albedo_init=0.5, emission_init=5.0):
    """edge^3 grid at `occupancy` (128^3 at 25%: ~524k voxels), 1% of the
    voxels emitters.  Learnable albedo starts at 0.5 and emitter radiance at
    5; the hidden target draws albedo U[0.1, 0.9] per voxel and channel and
    radiance U[1, 10] per emitter and channel from `target_seed`.  Camera
    outside the grid's corner looking at its centre, 60 degree vertical FOV."""
    sc = scenes.random_grid_scene(edge, occupancy, emissive_fraction=emissive_fraction, seed=seed)
    n = sc.aabbs.shape[0]
    emit = np.full(n, -1, np.int32)
    light_prims = sc.cube_lights["primitive_id"].astype(np.int64)
    emit[light_prims] = np.arange(light_prims.shape[0], dtype=np.int32)
    rng = np.random.default_rng(target_seed)
    a_t = rng.uniform(0.1, 0.9, (n, 3)).astype(np.float32)
    e_t = rng.uniform(1.0, 10.0, (light_prims.shape[0], 3)).astype(np.float32)
    half = edge * 0.5
    iv, ip = scenes.camera_matrices((-half * 0.5, float(edge), -half * 0.5), (half, half, half), width, height,
                                    fovy_deg=60.0)
    return AdjointScene(sc, emit, a_t, e_t, np.full((n, 3), albedo_init, np.float32),
                        np.full((light_prims.shape[0], 3), emission_init, np.float32), iv, ip, width, height)


class AdjointRenderer:
    """ct_adjoint_forward / ct_adjoint_backward over one AdjointScene on the
    current CUDA device and stream.  Parameters and images are torch tensors
    on the device: albedo (n_prim, 3), emission (n_emit, 3), image
    (H, W, 3)."""

    def __init__(self, ascene, spp=64, max_depth=3, seed=1, device="cuda", miss_radiance=0.0):
        self.a = ascene
        sc = ascene.scene
        self.device = device
        self.instances = _dev(sc.instances, device)
        self.aabbs = _dev(sc.aabbs, device)
        self.accel = Accel(self.instances, sc.instances.shape[0], self.aabbs, sc.aabbs.shape[0], sc.voxel_extent)
        self.emitter_index = torch.from_numpy(ascene.emitter_index).to(device)
        cam = np.zeros(1, L.CAMERA_VIEW)
        cam["inv_view"], cam["inv_proj"] = ascene.inv_view, ascene.inv_proj
        self.camera = _dev(cam, device)
        self.n_prim = sc.aabbs.shape[0]
        self.n_emit = ascene.emission_target.shape[0]
        self.W, self.H = ascene.width, ascene.height
        self.spp, self.max_depth, self.seed = spp, max_depth, seed
        self.miss_radiance = miss_radiance

    def desc(self, rect=None, f64=False, spp=None):
        d = native.AdjointDesc()
        d.struct_size = ctypes.sizeof(native.AdjointDesc)
        d.width, d.height = self.W, self.H
        d.spp = self.spp if spp is None else spp
        d.max_depth = self.max_depth
        d.seed = self.seed
        d.flags = native.CT_ADJOINT_IMAGE_F64 if f64 else 0
        d.primitive_count = self.n_prim
        d.emitter_count = self.n_emit
        if rect is not None:
            for i in range(4):
                d.rect[i] = rect[i]
        d.miss_radiance = self.miss_radiance
        d.camera_address = self.camera.data_ptr()
        d.emitter_index_address = self.emitter_index.data_ptr()
        return d

    @staticmethod
    def _stream():
        return torch.cuda.current_stream().cuda_stream

    def forward(self, albedo, emission, rect=None, f64=False, spp=None):
        """The image (H, W, 3), float32 (or float64 with f64); pixels outside
        rect are zero."""
        albedo = albedo.contiguous()
        emission = emission.contiguous()
        img = torch.zeros((self.H, self.W, 3), dtype=torch.float64 if f64 else torch.float32, device=self.device)
        d = self.desc(rect, f64, spp)
        native.check("ct_adjoint_forward", native.lib().ct_adjoint_forward(
            self.accel.handle, ctypes.byref(d), albedo.data_ptr(), emission.data_ptr(), img.data_ptr(),
            self._stream()))
        return img

    def backward(self, albedo, emission, d_image, rect=None, spp=None):
        """(d_albedo, d_emission): the gradient of a loss whose derivative
        with respect to the image is d_image (H, W, 3)."""
        albedo = albedo.contiguous()
        emission = emission.contiguous()
        d_image = d_image.to(torch.float32).contiguous()
        ga = torch.zeros_like(albedo)
        ge = torch.zeros_like(emission)
        d = self.desc(rect, False, spp)
        native.check("ct_adjoint_backward", native.lib().ct_adjoint_backward(
            self.accel.handle, ctypes.byref(d), albedo.data_ptr(), emission.data_ptr(), d_image.data_ptr(),
            ga.data_ptr(), ge.data_ptr(), self._stream()))
        return ga, ge

    def close(self):
        self.accel.free()
