// ct_adjoint.cuh -- path-replay adjoint of a plain path tracer over
// per-voxel albedo and emission (ct_adjoint_forward / ct_adjoint_backward,
// include/ct.h).  Compiled with ct_kernels.cu: it uses the library's walk,
// hit geometry and scatter sampling (ct_pt.cuh) and its device status word.
//
// The forward model, per sample of a pixel: a camera ray jittered inside
// the pixel, then up to max_depth closest-voxel hits (intersect()'s rules,
// bounce.glsl:9-125).  A hit voxel adds its emission times the throughput;
// a bounce leaves from the hit point moved off the surface twice
// (compute_ray_origin, primitives.glsl:233-257) in a cosine-weighted
// direction (random_cosine_direction, prng.glsl:84-106), so the Lambertian
// f cos / pdf (mat.glsl:66-88, light.glsl:200-229) is the voxel's albedo.
//
// The backward pass replays every path from its RNG counters (pixel,
// sample, frame seed): geometry does not depend on albedo or emission, so
// the replay meets the same vertices.  It keeps the path's vertices in
// registers only while it gathers the suffix radiance S_k from the end of
// the path back to the camera, then adds the gradients with atomics.
//
// One thread per pixel walks its samples in order, so the forward image is
// the same sum in the same order on every run.

namespace ct_adjoint {

struct Desc {
  uint32_t W, H, spp, max_depth, seed, n_prim, n_emit, x0, y0, x1, y1;
  const ct_camera_view *cam;
  const int32_t *emitter_index;
};

// the camera's matrices, loaded once per block
struct Camera {
  m4 inv_view, inv_proj;
};
__device__ __forceinline__ void load_camera(const Desc &D, Camera &C) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    C.inv_view = load_m4(D.cam->inv_view);
    C.inv_proj = load_m4(D.cam->inv_proj);
  }
  __syncthreads();
}

// the camera ray of rgen.glsl:18-42 with the pixel centre moved by (jx, jy)
// in [0, 1) instead of 0.5
__device__ __forceinline__ void camera_ray_jittered(const Desc &D, const Camera &C, uint32_t x, uint32_t y, float jx,
                                                    float jy, f3 &o, f3 &d) {
  const f2 pixel = f2{(float)x, (float)y} + f2{jx, jy};
  const f2 inv_uv = pixel / f2{(float)D.W, (float)D.H};
  const f2 dd = inv_uv * 2.0f - 1.0f;
  o = xyz(mul(C.inv_view, mk4(0.f, 0.f, 0.f, 1.f)));
  const f4 target = mul(C.inv_proj, mk4(dd.x, dd.y, 1.f, 1.f));
  d = xyz(mul(C.inv_view, mk4(normalize(xyz(target)), 0.f)));
}

// closest voxel of intersect() along (o, d); the global primitive index,
// hit point and normal of that voxel
__device__ __forceinline__ bool closest_voxel(const DevAccel &A, f3 o, f3 d, uint32_t pixel, RayStats &rs,
                                              uint32_t &gprim, f3 &pos, f3 &nrm) {
  ClosestWalk w;
  const auto ray = [&](f3 &ro, f3 &rd) { ro = o; rd = d; };
  if (!closest_walk_begin(A, w, o, d))
    while (closest_walk_advance(A, w, 1 << 20, pixel, rs, ray) == DDA_MORE) {
    }
  if (!w.best.hit) return false;
  gprim = w.best.gprim;
  bounce_geometry(A, o, d, w.best.inst, w.best.prim, w.best.gprim, pos, nrm);
  return true;
}

// the vertices of sample s of pixel (x, y): their global primitive indices,
// n of them (a path ends at max_depth vertices or at a miss)
__device__ __forceinline__ uint32_t trace_path(const DevAccel &A, const Desc &D, const Camera &C, uint32_t x,
                                               uint32_t y, uint32_t s, RayStats &rs, uint32_t *verts) {
  const uint32_t pixel = y * D.W + x;
  uint32_t seed = tea(pixel, D.seed + s);
  const float jx = rnd(seed);
  const float jy = rnd(seed);
  f3 o, d;
  camera_ray_jittered(D, C, x, y, jx, jy, o, d);
  uint32_t n = 0;
  for (uint32_t k = 0; k < D.max_depth; k++) {
    uint32_t g;
    f3 pos, nrm;
    rs.bounce++;
    if (!closest_voxel(A, o, d, pixel, rs, g, pos, nrm)) break;
    verts[n++] = g;
    if (k + 1 == D.max_depth) break;
    o = offset_twice(pos, nrm);
    d = random_cosine_direction(seed, nrm);
    if (normal_near_zero(d)) d = nrm;
  }
  return n;
}

__device__ __forceinline__ f3 albedo_of(const float *albedo, uint32_t g) {
  return f3{__ldg(&albedo[3u * g]), __ldg(&albedo[3u * g + 1u]), __ldg(&albedo[3u * g + 2u])};
}
__device__ __forceinline__ bool emission_of(const Desc &D, const float *emission, uint32_t g, f3 &e) {
  const int32_t slot = __ldg(&D.emitter_index[g]);
  if (slot < 0 || (uint32_t)slot >= D.n_emit) return false;
  e = f3{__ldg(&emission[3u * slot]), __ldg(&emission[3u * slot + 1u]), __ldg(&emission[3u * slot + 2u])};
  return true;
}

// Forward: image[p] = (1/spp) sum_s sum_k T_k E[v_k].  Real is the type of
// the throughput and sums (float for rendering, double for the finite
// differences of a gradient check).
template <class Real>
__global__ void __launch_bounds__(128) k_adjoint_forward(DevAccel A, Desc D, const float *albedo,
                                                         const float *emission, Real *image) {
  __shared__ Camera C;
  load_camera(D, C);
  const uint32_t x = D.x0 + blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = D.y0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= D.x1 || y >= D.y1) return;
  RayStats rs = {};
  uint32_t verts[CT_ADJOINT_MAX_DEPTH];
  Real sx = 0, sy = 0, sz = 0;
  for (uint32_t s = 0; s < D.spp; s++) {
    const uint32_t n = trace_path(A, D, C, x, y, s, rs, verts);
    Real tx = 1, ty = 1, tz = 1, lx = 0, ly = 0, lz = 0;
    for (uint32_t k = 0; k < n; k++) {
      f3 e;
      if (emission_of(D, emission, verts[k], e)) {
        lx = lx + tx * (Real)e.x;
        ly = ly + ty * (Real)e.y;
        lz = lz + tz * (Real)e.z;
      }
      const f3 a = albedo_of(albedo, verts[k]);
      tx = tx * (Real)a.x;
      ty = ty * (Real)a.y;
      tz = tz * (Real)a.z;
    }
    sx = sx + lx;
    sy = sy + ly;
    sz = sz + lz;
  }
  const uint32_t p = 3u * (y * D.W + x);
  const Real inv = (Real)1 / (Real)D.spp;
  image[p] = sx * inv;
  image[p + 1] = sy * inv;
  image[p + 2] = sz * inv;
}

// Backward: replays each path, gathers S_k from the last vertex back, adds
// g T_k S_k to d_albedo[v_k] and g T_k to d_emission[slot of v_k].
__global__ void __launch_bounds__(128) k_adjoint_backward(DevAccel A, Desc D, const float *albedo,
                                                          const float *emission, const float *d_image,
                                                          float *d_albedo, float *d_emission) {
  __shared__ Camera C;
  load_camera(D, C);
  const uint32_t x = D.x0 + blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = D.y0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= D.x1 || y >= D.y1) return;
  const uint32_t p = 3u * (y * D.W + x);
  const float inv = 1.0f / (float)D.spp;
  const f3 g = f3{d_image[p] * inv, d_image[p + 1] * inv, d_image[p + 2] * inv};
  if (g.x == 0.f && g.y == 0.f && g.z == 0.f) return;
  RayStats rs = {};
  uint32_t verts[CT_ADJOINT_MAX_DEPTH];
  for (uint32_t s = 0; s < D.spp; s++) {
    const uint32_t n = trace_path(A, D, C, x, y, s, rs, verts);
    if (n == 0) continue;
    // T_k for every vertex, front to back
    f3 T[CT_ADJOINT_MAX_DEPTH];
    f3 t = mk3(1.f);
    for (uint32_t k = 0; k < n; k++) {
      T[k] = t;
      t = t * albedo_of(albedo, verts[k]);
    }
    // S_k back to front: S_{n-1} = 0, S_k = a[v_{k+1}] S_{k+1} + E[v_{k+1}]
    f3 S = mk3(0.f);
    for (int k = (int)n - 1; k >= 0; k--) {
      const uint32_t v = verts[k];
      const f3 gt = g * T[k];
      f3 e;
      const bool emits = emission_of(D, emission, v, e);
      if (emits) {
        const int32_t slot = __ldg(&D.emitter_index[v]);
        atomicAdd(&d_emission[3u * slot], gt.x);
        atomicAdd(&d_emission[3u * slot + 1u], gt.y);
        atomicAdd(&d_emission[3u * slot + 2u], gt.z);
      }
      if (k + 1 < (int)n) {
        const f3 ga = gt * S;
        atomicAdd(&d_albedo[3u * v], ga.x);
        atomicAdd(&d_albedo[3u * v + 1u], ga.y);
        atomicAdd(&d_albedo[3u * v + 2u], ga.z);
      }
      // the radiance gathered after v_{k-1}: this vertex's albedo times what
      // it gathers, plus its emission
      S = albedo_of(albedo, v) * S + (emits ? e : mk3(0.f));
    }
  }
}

}  // namespace ct_adjoint

static ct_adjoint::Desc adjoint_desc(const ct_adjoint_desc &d) {
  ct_adjoint::Desc D;
  D.W = d.width;
  D.H = d.height;
  D.spp = d.spp;
  D.max_depth = d.max_depth;
  D.seed = d.seed;
  D.n_prim = d.primitive_count;
  D.n_emit = d.emitter_count;
  const bool whole = d.rect[2] == 0;
  D.x0 = whole ? 0u : d.rect[0];
  D.y0 = whole ? 0u : d.rect[1];
  D.x1 = whole ? d.width : d.rect[2];
  D.y1 = whole ? d.height : d.rect[3];
  D.cam = (const ct_camera_view *)(uintptr_t)d.camera_address;
  D.emitter_index = (const int32_t *)(uintptr_t)d.emitter_index_address;
  return D;
}

cudaError_t ct_launch_adjoint(const DevAccel &A, const ct_adjoint_desc &d, const float *albedo, const float *emission,
                              void *image, const float *d_image, float *d_albedo, float *d_emission, int backward,
                              cudaStream_t s) {
  const ct_adjoint::Desc D = adjoint_desc(d);
  const dim3 blk(16, 8);
  const dim3 grid((D.x1 - D.x0 + blk.x - 1) / blk.x, (D.y1 - D.y0 + blk.y - 1) / blk.y);
  if (grid.x == 0 || grid.y == 0) return cudaSuccess;
  if (backward) {
    CT_TIMED(CT_K_ADJOINT_BACKWARD, s,
             ct_adjoint::k_adjoint_backward<<<grid, blk, 0, s>>>(A, D, albedo, emission, d_image, d_albedo,
                                                                d_emission));
  } else if (d.flags & CT_ADJOINT_IMAGE_F64) {
    CT_TIMED(CT_K_ADJOINT_FORWARD, s,
             ct_adjoint::k_adjoint_forward<double><<<grid, blk, 0, s>>>(A, D, albedo, emission, (double *)image));
  } else {
    CT_TIMED(CT_K_ADJOINT_FORWARD, s,
             ct_adjoint::k_adjoint_forward<float><<<grid, blk, 0, s>>>(A, D, albedo, emission, (float *)image));
  }
  return cudaGetLastError();
}
