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
  float miss;  // radiance of rays that leave the scene
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
  NoObjRay R;
  const auto ray = [&](f3 &ro, f3 &rd) { ro = o; rd = d; };
  if (!closest_walk_begin(A, w, o, d, R))
    while (closest_walk_advance(A, w, 1 << 20, pixel, rs, ray, R) == DDA_MORE) {
    }
  if (!w.best.hit) return false;
  gprim = w.best.gprim;
  bounce_geometry(A, o, d, w.best.inst, w.best.prim, w.best.gprim, pos, nrm);
  return true;
}

// the vertices of sample s of pixel (x, y): their global primitive indices,
// n of them (a path ends at max_depth vertices or at a miss; `missed` tells
// which)
__device__ __forceinline__ uint32_t trace_path(const DevAccel &A, const Desc &D, const Camera &C, uint32_t x,
                                               uint32_t y, uint32_t s, RayStats &rs, uint32_t *verts,
                                               bool &missed) {
  const uint32_t pixel = y * D.W + x;
  uint32_t seed = tea(pixel, D.seed + s);
  const float jx = rnd(seed);
  const float jy = rnd(seed);
  f3 o, d;
  camera_ray_jittered(D, C, x, y, jx, jy, o, d);
  uint32_t n = 0;
  missed = false;
  for (uint32_t k = 0; k < D.max_depth; k++) {
    uint32_t g;
    f3 pos, nrm;
    rs.bounce++;
    if (!closest_voxel(A, o, d, pixel, rs, g, pos, nrm)) {
      missed = true;
      break;
    }
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
    bool missed;
    const uint32_t n = trace_path(A, D, C, x, y, s, rs, verts, missed);
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
    if (missed && D.miss != 0.f) {
      lx = lx + tx * (Real)D.miss;
      ly = ly + ty * (Real)D.miss;
      lz = lz + tz * (Real)D.miss;
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
    bool missed;
    const uint32_t n = trace_path(A, D, C, x, y, s, rs, verts, missed);
    if (n == 0) continue;
    // T_k for every vertex, front to back
    f3 T[CT_ADJOINT_MAX_DEPTH];
    f3 t = mk3(1.f);
    for (uint32_t k = 0; k < n; k++) {
      T[k] = t;
      t = t * albedo_of(albedo, verts[k]);
    }
    // S_k back to front: S_{n-1} = the miss light if the path left the
    // scene after v_{n-1}, else 0; S_k = a[v_{k+1}] S_{k+1} + E[v_{k+1}]
    f3 S = missed ? mk3(D.miss) : mk3(0.f);
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
      if (k + 1 < (int)n || missed) {
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

// ---------------------------------------------------------------------------
// Cache-terminated paths for the neural radiance cache (ct_nrc_trace): the
// sample-0 path of ct_adjoint_forward, stopped at surface vertex v_c
// (c = cache_vertex, v0 the primary hit).

struct NrcOut {
  float *base, *thp;
  ct_nrc_query *query;
  uint32_t train_paths, train_offset, train_bounces, cache_vertex;
  ct_nrc_query *tq;
  float *tpartial, *tthp;
};

__device__ __forceinline__ ct_nrc_query make_query(f3 pos, f3 dir, f3 nrm, f3 albedo) {
  ct_nrc_query q;
  q.position[0] = pos.x; q.position[1] = pos.y; q.position[2] = pos.z;
  q.direction[0] = dir.x; q.direction[1] = dir.y; q.direction[2] = dir.z;
  q.normal[0] = nrm.x; q.normal[1] = nrm.y; q.normal[2] = nrm.z;
  q.albedo[0] = albedo.x; q.albedo[1] = albedo.y; q.albedo[2] = albedo.z;
  return q;
}
__device__ __forceinline__ ct_nrc_query no_query() { return make_query(mk3(0.f), mk3(0.f), mk3(0.f), mk3(-1.f)); }

// The path of pixel (x, y) up to its cache vertex v_c: base radiance
// (emission at v0 .. v_{c-1}, or miss light), throughput to v_c, and the walk
// state there (seed, v_c's voxel, hit point, normal, incoming direction).
// false when the path ends before v_c.
struct CachePath {
  f3 base, thp, pos, nrm, dir;
  uint32_t seed, g;
};
__device__ bool trace_to_cache(const DevAccel &A, const Desc &D, const Camera &C, const float *albedo,
                               const float *emission, uint32_t x, uint32_t y, uint32_t cache_vertex, RayStats &rs,
                               CachePath &p) {
  const uint32_t pixel = y * D.W + x;
  p.seed = tea(pixel, D.seed);
  const float jx = rnd(p.seed);
  const float jy = rnd(p.seed);
  f3 o, d;
  camera_ray_jittered(D, C, x, y, jx, jy, o, d);
  p.base = mk3(0.f);
  p.thp = mk3(1.f);
  for (uint32_t k = 0;; k++) {
    uint32_t g;
    f3 pos, nrm;
    rs.bounce++;
    if (!closest_voxel(A, o, d, pixel, rs, g, pos, nrm)) {
      p.base = p.base + p.thp * mk3(D.miss);
      return false;
    }
    if (k == cache_vertex) {
      p.pos = pos;
      p.nrm = nrm;
      p.dir = d;
      p.g = g;
      return true;
    }
    f3 e;
    if (emission_of(D, emission, g, e)) p.base = p.base + p.thp * e;
    p.thp = p.thp * albedo_of(albedo, g);
    o = offset_twice(pos, nrm);
    d = random_cosine_direction(p.seed, nrm);
    if (normal_near_zero(d)) d = nrm;
  }
}

// one pixel's cache-terminated path
__device__ __forceinline__ void nrc_trace_pixel(const DevAccel &A, const Desc &D, const Camera &C, const float *albedo,
                                                const float *emission, const NrcOut &out, uint32_t x, uint32_t y) {
  RayStats rs = {};
  CachePath p;
  const uint32_t pixel = y * D.W + x;
  const bool cached = trace_to_cache(A, D, C, albedo, emission, x, y, out.cache_vertex, rs, p);
  st3(out.base + 3u * pixel, p.base);
  st3(out.thp + 3u * pixel, cached ? p.thp : mk3(0.f));
  out.query[pixel] = cached ? make_query(p.pos, -p.dir, p.nrm, albedo_of(albedo, p.g)) : no_query();
}

// self-training paths: the pixel's path again, past v_c for train_bounces
// more bounces
__device__ __forceinline__ void nrc_train_path(const DevAccel &A, const Desc &D, const Camera &C, const float *albedo,
                                               const float *emission, const NrcOut &out, uint32_t i) {
  const uint32_t px = D.W * D.H;
  const uint32_t stride = px / out.train_paths;
  const uint32_t pixel = (uint32_t)(((uint64_t)out.train_offset + (uint64_t)i * stride) % px);
  const uint32_t x = pixel % D.W, y = pixel / D.W;
  const uint32_t B = out.train_bounces;
  ct_nrc_query *tq = out.tq + (size_t)i * (B + 1u);
  RayStats rs = {};
  CachePath p;
  f3 E[8], a[8];
  uint32_t reached = 0;
  bool missed = false;
  if (trace_to_cache(A, D, C, albedo, emission, x, y, out.cache_vertex, rs, p)) {
    f3 pos = p.pos, nrm = p.nrm, d = p.dir;
    uint32_t g = p.g;
    for (uint32_t j = 0;; j++) {
      const f3 alb = albedo_of(albedo, g);
      tq[j] = make_query(pos, -d, nrm, alb);
      if (j == B) break;  // the terminal vertex: the cache bootstraps the rest
      f3 e;
      E[j] = emission_of(D, emission, g, e) ? e : mk3(0.f);
      a[j] = alb;
      reached = j + 1;
      const f3 o = offset_twice(pos, nrm);
      d = random_cosine_direction(p.seed, nrm);
      if (normal_near_zero(d)) d = nrm;
      rs.bounce++;
      if (!closest_voxel(A, o, d, pixel, rs, g, pos, nrm)) {
        missed = true;
        break;
      }
    }
  }
  // partial radiance and throughput from each reached vertex to the
  // terminal one, back to front
  f3 part = missed ? mk3(D.miss) : mk3(0.f);
  f3 thr = missed ? mk3(0.f) : mk3(1.f);
  for (int j = (int)B - 1; j >= 0; j--) {
    float *pp = out.tpartial + 3u * ((size_t)i * B + (uint32_t)j);
    float *tt = out.tthp + 3u * ((size_t)i * B + (uint32_t)j);
    if ((uint32_t)j >= reached) {
      tq[j] = no_query();
      st3(pp, mk3(0.f));
      st3(tt, mk3(0.f));
      continue;
    }
    part = E[j] + a[j] * part;
    thr = a[j] * thr;
    st3(pp, part);
    st3(tt, thr);
  }
  if (reached < B || missed) tq[B] = no_query();
}

// One launch for both: the first blocks take the self-training paths (each a
// long chain of walks, few of them), the others 128 pixels each, so that the
// pixels' paths fill the GPU while the training paths run.
__global__ void __launch_bounds__(128) k_nrc_trace(DevAccel A, Desc D, const float *albedo, const float *emission,
                                                   NrcOut out, uint32_t train_blocks) {
  __shared__ Camera C;
  load_camera(D, C);
  if (blockIdx.x < train_blocks) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < out.train_paths) nrc_train_path(A, D, C, albedo, emission, out, i);
    return;
  }
  const uint32_t pixel = (blockIdx.x - train_blocks) * blockDim.x + threadIdx.x;
  if (pixel >= D.W * D.H) return;
  nrc_trace_pixel(A, D, C, albedo, emission, out, pixel % D.W, pixel / D.W);
}

}  // namespace ct_adjoint

cudaError_t ct_launch_nrc_trace(const DevAccel &A, const ct_adjoint_desc &d, const float *albedo,
                                const float *emission, const ct_nrc_frame &f, cudaStream_t s) {
  ct_adjoint::Desc D;
  D.W = d.width;
  D.H = d.height;
  D.spp = 1;
  D.max_depth = f.cache_vertex;  // not read: the cache vertex ends the path
  D.seed = d.seed;
  D.n_prim = d.primitive_count;
  D.n_emit = d.emitter_count;
  D.x0 = D.y0 = 0;
  D.x1 = d.width;
  D.y1 = d.height;
  D.miss = d.miss_radiance;
  D.cam = (const ct_camera_view *)(uintptr_t)d.camera_address;
  D.emitter_index = (const int32_t *)(uintptr_t)d.emitter_index_address;
  ct_adjoint::NrcOut o;
  o.base = (float *)(uintptr_t)f.base_address;
  o.thp = (float *)(uintptr_t)f.throughput_address;
  o.query = (ct_nrc_query *)(uintptr_t)f.query_address;
  o.train_paths = f.train_paths;
  o.train_offset = f.train_offset;
  o.train_bounces = f.train_bounces;
  o.cache_vertex = f.cache_vertex;
  o.tq = (ct_nrc_query *)(uintptr_t)f.train_query_address;
  o.tpartial = (float *)(uintptr_t)f.train_partial_address;
  o.tthp = (float *)(uintptr_t)f.train_throughput_address;
  const uint32_t train_blocks = (f.train_paths + 127u) / 128u;
  const uint32_t pixel_blocks = (uint32_t)(((uint64_t)D.W * D.H + 127u) / 128u);
  CT_TIMED(CT_K_NRC_TRACE, s,
           ct_adjoint::k_nrc_trace<<<train_blocks + pixel_blocks, 128, 0, s>>>(A, D, albedo, emission, o,
                                                                                 train_blocks));
  return cudaGetLastError();
}

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
  D.miss = d.miss_radiance;
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
