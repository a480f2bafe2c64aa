// ct_kernels.cu -- per-pixel kernels of the frame: primary visibility,
// ReSTIR DI (RIS + temporal reuse; spatial reuse + shading) and TAA.
//
// One thread per pixel, 16x8-pixel blocks so that a warp covers a 16x2
// screen tile (neighbouring rays walk the same bricks).  Per-frame constants
// (camera matrices, table addresses) are read once per block into shared
// memory.  Buffers keep the reference's array-of-structs layout so that the
// caller's RESTIR/WORLD tables are used in place.
#include <cuda_runtime.h>
#include "ct_device.cuh"
#include <cstddef>
#include "ct_kernels.cuh"
#include "ct_profile.cuh"

// ---------------------------------------------------------------------------
// per-block frame constants
struct BlockConsts {
  FrameView F;
  m4 inv_view, inv_proj, inv_prev_mvp;
};

__device__ void load_frame_view(const ct_push_constant &pc, BlockConsts &B) {
  FrameView &F = B.F;
  const ct_world *w = (const ct_world *)(uintptr_t)pc.world_buffer;
  const ct_restir *r = (const ct_restir *)(uintptr_t)pc.restir_buffer;
  const ct_status_block *s = (const ct_status_block *)(uintptr_t)pc.status_buffer;
  const ct_camera_view *c = (const ct_camera_view *)(uintptr_t)pc.camera_buffer;
  F.W = pc.size[0];
  F.H = pc.size[1];
  F.instances = (const ct_instance *)(uintptr_t)w->instance_address;
  F.instances_prev = (const ct_instance *)(uintptr_t)w->instance_address_prev;
  F.primitives = (const ct_primitive *)(uintptr_t)w->primitive_address;
  F.aabbs = (const ct_aabb *)(uintptr_t)w->aabb_address;
  F.remap_p = (const uint32_t *)(uintptr_t)w->remapped_primitive_address;
  F.remap_l = (const uint32_t *)(uintptr_t)w->remapped_cube_light_address;
  F.materials = (const ct_material *)(uintptr_t)w->material_address;
  F.point_lights = (const ct_light *)(uintptr_t)w->point_light_address;
  F.cube_lights = (const ct_light *)(uintptr_t)w->cube_light_address;
  F.env_lights = (const ct_light *)(uintptr_t)w->env_light_address;
  F.prev_reservoir = (ct_reservoir *)(uintptr_t)r->previous_reservoir_address;
  F.int_reservoir = (ct_reservoir *)(uintptr_t)r->intermediate_reservoir_address;
  F.cur_reservoir = (ct_reservoir *)(uintptr_t)r->reservoir_address;
  F.prev_di = (ct_di_info *)(uintptr_t)r->previous_di_address;
  F.di = (ct_di_info *)(uintptr_t)r->di_address;
  F.velocity = (ct_velocity *)(uintptr_t)r->velocity_address;
  F.out_path_reservoir = (ct_path_reservoir *)(uintptr_t)r->output_path_reservoir_address;
  F.temporal_path_reservoir = (ct_path_reservoir *)(uintptr_t)r->temporal_path_reservoir_address;
  F.indirect_color = (float *)(uintptr_t)r->indirect_color_address;
  F.swapchain = (float4 *)pc.swapchain;
  F.previous_swapchain = (const float4 *)pc.previous_swapchain;
  F.taa_frame = (float4 *)pc.taa_frame;
  F.frame_number = s->frame_number;
  F.is_active = s->is_active;
  F.obj_count = s->obj_count;
  F.is_afternoon = s->is_afternoon;
  F.max_depth = s->max_depth;
  F.time = s->time;
  F.light_config = *(const ct_light_config *)(uintptr_t)s->light_config_address;
  F.camera = c;
  B.inv_view = load_m4(c->inv_view);
  B.inv_proj = load_m4(c->inv_proj);
  // inverse(prev_inv_proj) * inverse(prev_inv_view) (motion_vectors.glsl:78)
  B.inv_prev_mvp = mul(ct_inverse(load_m4(c->prev_inv_proj)), ct_inverse(load_m4(c->prev_inv_view)));
}

// get_ray_from_current_pixel (rgen.glsl:18-42), no jitter
__device__ __forceinline__ void camera_ray(const BlockConsts &B, uint32_t x, uint32_t y, f3 &o, f3 &d) {
  f2 pixel_center = (f2{(float)x, (float)y} + f2{0.0f, 0.0f}) + f2{0.5f, 0.5f};
  f2 inv_uv = pixel_center / f2{(float)B.F.W, (float)B.F.H};
  f2 dd = inv_uv * 2.0f - 1.0f;
  f4 origin = mul(B.inv_view, mk4(0.f, 0.f, 0.f, 1.f));
  o = xyz(origin);
  f4 target = mul(B.inv_proj, mk4(dd.x, dd.y, 1.f, 1.f));
  d = xyz(mul(B.inv_view, mk4(normalize(xyz(target)), 0.f)));
}

__device__ __forceinline__ void count_rays(const ct_params &P, const RayStats &rs) {
  if (!(P.flags & CT_PARAM_COUNT_RAYS) || P.counters_address == 0) return;
  unsigned long long *c = (unsigned long long *)(uintptr_t)P.counters_address;
  // every thread of the block reaches this point (kernels do not return early)
  const unsigned mask = 0xFFFFFFFFu;
  const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
  const int leader = 0;
  const uint32_t v[CT_COUNTER_COUNT] = {rs.primary,    rs.shadow,     rs.bounce,   rs.voxel_tests, rs.bricks,
                                        rs.candidates, rs.neighbours, rs.temporal, rs.hits,        rs.bounce_hits,
                                        rs.walker_bricks};
#pragma unroll
  for (int i = 0; i < CT_COUNTER_COUNT; i++) {
    uint32_t t = __reduce_add_sync(mask, v[i]);
    if (lane == leader && t) atomicAdd(&c[i], (unsigned long long)t);
  }
}

__device__ __forceinline__ void pixel_of(uint32_t &x, uint32_t &y) {
  x = blockIdx.x * blockDim.x + threadIdx.x;
  y = blockIdx.y * blockDim.y + threadIdx.y;
}

// ---------------------------------------------------------------------------
// pass 1, front half: primary visibility (rgen.glsl:46-201, 319) with the
// closest-hit shader (rchit.glsl:18-54) and miss shader (rmiss.glsl:25-28)
// 10 blocks of 128 per SM (48 registers, spills to L1): 0.97 ms per 1080p
// frame against 1.02 ms at 8 blocks (64 registers), 1.09 ms at 6 and 1.07
// ms when the register count is left free
#ifndef CT_PRIMARY_MIN_BLOCKS
#define CT_PRIMARY_MIN_BLOCKS 10
#endif
__global__ void __launch_bounds__(128, CT_PRIMARY_MIN_BLOCKS) k_trace_primary(ct_push_constant pc, DevAccel A, ct_params P) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  if (x < F.W && y < F.H) {
    const uint32_t screen_pos = y * F.W + x;
    const uint32_t seed = tea(y * F.W + x, F.frame_number);
    f3 o, d;
    camera_ray(B, x, y, o, d);
    rs.primary = 1;
    HitRecord h = trace_primary(A, o, d, 0.0f, 1e9f, screen_pos, rs);
    ct_di_info di;
    di.seed = seed;
    st3(di.ray_origin, o);
    di.confidence = 1.0f;
    if (h.hit) {
      rs.hits = 1;
      const DevGrid &g = A.grids[h.inst];
      // rchit model matrix as written in rchit.glsl:29-33 (column 1 takes
      // element [0][1] where [1][0] belongs)
      const m4 &T = g.obj2world_tlas;
      m4 model;
      model.c[0] = f4{T.c[0].x, T.c[0].y, T.c[0].z, 0.f};
      model.c[1] = f4{T.c[0].y, T.c[1].y, T.c[1].z, 0.f};
      model.c[2] = f4{T.c[2].x, T.c[2].y, T.c[2].z, 0.f};
      model.c[3] = f4{T.c[3].x, T.c[3].y, T.c[3].z, 1.f};
      f3 world_pos = o + d * h.t;
      const uint32_t first = F.instances[h.inst].first_primitive_index;
      const uint32_t actual = first != 0xFFFFFFFFu ? first + h.prim : first;
      const ct_aabb &bb = F.aabbs[actual];
      f3 center = (ld3(bb.minimum) + ld3(bb.maximum)) * 0.5f;
      center = xyz(mul(model, mk4(center, 1.f)));
      f3 nrm = cube_like_normal(normalize(world_pos - center));
      float dist = length(world_pos - o);
      uint32_t mat_index = F.primitives[actual].material_index;
      st3(di.position, world_pos);
      di.distance = dist;
      st3(di.normal, nrm);
      di.instance_hit.instance_id = h.inst;
      di.instance_hit.primitive_id = h.prim;
      di.mat_index = mat_index;
      // motion vector (motion_vectors.glsl:70-89)
      m4 obj2world = load_m4(F.instances[h.inst].transform);
      m4 prev_model = load_m4(F.instances_prev[h.inst].transform);
      m4 geometry_T = mul(prev_model, ct_inverse(obj2world));
      f4 prev_S = mul(mul(B.inv_prev_mvp, geometry_T), mk4(world_pos, 1.0f));
      f2 xi1 = f2{prev_S.x, prev_S.y} / prev_S.w;
      xi1 = 0.5f * xi1 + 0.5f;
      f2 xi = f2{(float)x, (float)y} + 0.5f;
      f2 mv = xi1 * f2{(float)F.W, (float)F.H} - xi;
      F.velocity[screen_pos].velocity[0] = mv.x;
      F.velocity[screen_pos].velocity[1] = mv.y;
    } else {
      f3 hv = f3{1.0f, 1.0f, 1.0f} * sky_color(F.time, F.is_afternoon, d);
      float4 px = make_float4(hv.x, hv.y, hv.z, 1.0f);
      F.swapchain[screen_pos] = px;
      if (F.is_active & CT_TAA_BIT) F.taa_frame[screen_pos] = px;
      if (P.flags & CT_PARAM_INDIRECT) st3(F.indirect_color + 3u * screen_pos, mk3(0.f));
      st3(di.position, mk3(0.f));
      di.distance = -1.0f;
      st3(di.normal, mk3(0.f));
      di.instance_hit.instance_id = CT_MAX_INSTANCES;
      di.instance_hit.primitive_id = CT_MAX_PRIMITIVES;
      di.mat_index = 0;
    }
    F.di[screen_pos] = di;
  }
  count_rays(P, rs);
}

// ---------------------------------------------------------------------------
// Scratch of the wavefront passes (see ct_workspace_size)
struct Workspace {
  RayQueue q;
  uint8_t *vis;    // [pixel * CT_VIS_SLOTS + slot] shadow-ray answers
  float *rad;      // [3 * (pixel * CT_VIS_SLOTS + slot)] radiance if visible
  uint32_t *nbr;   // [pixel * CT_MAX_NEIGHBORS + i] chosen neighbours
  uint2 *smeta;    // [pixel] (neighbour count, seed after the choice)
};

// BRDF-sampled candidates of RIS (restir_resampling.glsl:193-248): per
// candidate one scatter direction from the material's callable
// (sample_material, light.glsl:231-270), a closest hit along it
// (intersect(), bounce.glsl:9-125) and, when that voxel emits, the
// candidate's contribution with the MIS weight of both strategies; the light
// index is the hit primitive's PRIMITIVE.light_index.
struct BrdfCandidates {
  Reservoir res;
  uint32_t seed;
  bool moved;  // a callable changed the hit point or normal
};
__device__ BrdfCandidates ris_brdf_candidates(const FrameView &F, const DevAccel &A, f3 ray_origin, f3 ray_dir,
                                              Shade S, uint32_t seed, uint32_t nee, uint32_t n_brdf,
                                              uint32_t cube_count, float extent,
                                              uint32_t pixel);  // defined after the PT pieces

// RIS over the active light types (restir_resampling.glsl:19-255), without
// the final visibility pass.  Candidates are evaluated with visibility off.
// `requires_visibility` is false when the BRDF candidates' reservoir wins
// the final merge (the shader then skips reservoir_visibility_pass).
template <bool BRDF>
__device__ Reservoir ris_candidates(const FrameView &F, const DevAccel &A, const ct_params &P, f3 ray_origin,
                                    f3 ray_dir, const Shade &S, const Material &mat, float confidence, uint32_t &seed,
                                    uint32_t pixel, bool &requires_visibility, RayStats &rs) {
  requires_visibility = true;
  confidence = gclamp(confidence, 0.0f, 1.0f);
  const bool point_active = (F.is_active & CT_RIS_POINT_LIGHT_BIT) != 0;
  const bool env_active = (F.is_active & CT_RIS_ENV_LIGHT_BIT) != 0;
  const bool cube_active = (F.is_active & CT_RIS_CUBE_LIGHT_BIT) != 0;
  const ct_light_config &lc = F.light_config;
  const uint32_t point_count = lc.point_light_count;
  const uint32_t n_point = gmax(f2u(gmin((float)P.max_ris_point_samples * (1.0f - confidence), (float)point_count)),
                                P.min_ris_point_samples);
  const uint32_t env_count = lc.env_map_count;
  const uint32_t n_env = gmax(f2u(gmin((float)P.max_ris_env_samples * (1.0f - confidence), (float)env_count)),
                              P.min_ris_env_samples);
  const uint32_t cube_count = lc.cube_light_count < 1 ? 1u : lc.cube_light_count;
  const uint32_t n_cube = gmax(f2u(gmin((float)P.max_ris_cube_samples * (1.0f - confidence), (float)cube_count)),
                               P.min_ris_cube_samples);
  const uint32_t n_brdf = lc.brdf_count + n_env;
  const uint32_t nee = n_point + n_cube;
  f3 scatter_dir = mk3(0.f);
  const f3 neg_dir = -ray_dir;
  VisNever never;
  Reservoir res = reservoir_empty();

  // rng_count: the count the shader draws the index from (the cube count is
  // clamped to >= 1, restir_resampling.glsl:51-52); a light buffer with no
  // entries yields a zero light, which contributes nothing.
  auto candidate = [&](Reservoir &dst, const ct_light *buf, uint32_t rng_count, uint32_t real_count, uint32_t type,
                       float pdf) {
    uint32_t li = gmin(urnd_interval(seed, 0u, rng_count), rng_count - 1u);
    Light light;
    if (li >= real_count) { light = Light{}; light.type = type; } else light = load_light(buf, li);
    float light_pdf = 1.0f, G;
    uint32_t current_seed = seed;
    rs.candidates++;
    f3 Fv = calculate_sampled_light(F, ray_dir, S.P, S.n, S.inst, S.prim, mat, light, pdf, light_pdf, G, seed, true,
                                    false, false, scatter_dir, pixel, never, 0u);
    float brdf_pdf = sample_material_pdf(mat, S.n, neg_dir, scatter_dir) * G;
    float m_i = 1.0f / gmax((float)nee * light_pdf + (float)n_brdf * brdf_pdf, 1e-6f);
    float w_i = luminance(Fv) * m_i;
    update_reservoir(dst, li, type, current_seed, Fv, w_i, 1.0f, seed);
  };

  if (point_active) {
    float pdf = 1.0f / (float)point_count;
    for (uint32_t l = 0; l < n_point; l++) candidate(res, F.point_lights, point_count, point_count, CT_LIGHT_POINT, pdf);
  }
  if (env_active) {
    Reservoir er = reservoir_empty();
    float pdf = 1.0f / (float)env_count;
    for (uint32_t l = 0; l < n_env; l++) candidate(er, F.env_lights, env_count, env_count, CT_LIGHT_ENV_MAP, pdf);
    update_reservoir(res, er.Y, er.l_type, er.seed, er.F, er.W_sum, er.M, seed);
  }
  if (cube_active) {
    Reservoir cr = reservoir_empty();
    float pdf = 1.0f / (float)cube_count;
    for (uint32_t l = 0; l < n_cube; l++)
      candidate(cr, F.cube_lights, cube_count, lc.cube_light_count, CT_LIGHT_CUBE, pdf);
    update_reservoir(res, cr.Y, cr.l_type, cr.seed, cr.F, cr.W_sum, cr.M, seed);
  }
  if constexpr (BRDF) {
    const BrdfCandidates b =
        ris_brdf_candidates(F, A, ray_origin, ray_dir, S, seed, nee, n_brdf, cube_count, P.voxel_extent, pixel);
    seed = b.seed;
    // the rest of the first pass applies the same turn by turn_after_ris
    Shade St = S;
    turn_after_ris(F, St, ray_dir);
    const bool turned = St.P.x != S.P.x || St.P.y != S.P.y || St.P.z != S.P.z || St.n.x != S.n.x ||
                        St.n.y != S.n.y || St.n.z != S.n.z;
    if (b.moved != turned) ct_latch_error(CT_ERR_UNSUPPORTED, 43, pixel);
    if (update_reservoir(res, b.res.Y, b.res.l_type, b.res.seed, b.res.F, b.res.W_sum, b.res.M, seed))
      requires_visibility = false;
  }
  return res;
}

// answer-slot marker: RIS needs no visibility pass (BRDF candidate chosen)
#define CT_VIS_SKIP 2u

// reservoir_visibility_pass (reservoir.glsl:114-126); slot 0
template <class VP>
__device__ void ris_visibility(const FrameView &F, Reservoir &res, const Shade &S, uint32_t pixel, VP &vp) {
  bool visible = false;
  if (reservoir_valid(res)) {
    Light light = light_get_by_type(F, res.l_type, res.Y);
    uint32_t s2 = res.seed;
    float l_pdf = 1.0f;
    LightSample ls = sample_lights(F, S.P, S.n, S.inst, S.prim, light, l_pdf, s2, false, true, pixel, vp, 0u);
    visible = ls.vis;
  }
  res.W_y = visible ? (res.W_sum / luminance(res.F)) : 0.0f;
  res.F = res.F * (visible ? 1.0f : 0.0f);
}

// The previous frame's reservoir a pixel reprojects to
// (GATHER_TEMPORAL_RESERVOIR, restir_resampling.glsl:269-309)
struct Temporal {
  Reservoir prev;
  uint32_t prev_index;
  float confidence;
};
__device__ __forceinline__ Temporal gather_temporal(const FrameView &F, const ct_params &P, uint32_t x, uint32_t y,
                                                    uint32_t screen_pos) {
  Temporal T;
  f2 xi = f2{(float)x, (float)y} + 0.5f;
  f2 v = f2{F.velocity[screen_pos].velocity[0], F.velocity[screen_pos].velocity[1]};
  f2 xi1 = xi + v;
  const uint32_t px = f2u(xi1.x), py = f2u(xi1.y);
  T.prev_index = px + py * F.W;
  T.prev = reservoir_empty();
  if (T.prev_index < F.W * F.H) T.prev = load_reservoir(F.prev_reservoir, T.prev_index);
  const float predicted = gclamp(T.prev.M / P.max_influence_from_the_past, 0.0f, 1.0f);
  T.confidence = (T.prev.W_y > 0.0f) ? predicted : 0.0f;
  return T;
}

// TEMPORAL_REUSE (restir_resampling.glsl:311-416).  Shadow rays: slot 2 =
// current sample at the previous pixel, slot 1 = previous sample at the
// current pixel.  With `emit_only` the function stops after asking for the
// rays it needs (ray A only: ray B is asked for by temporal_prev_sample_ray).
// With CT_REMAP_BIT (a frame after a scene edit) the previous DI record's
// primitive and the previous reservoir's cube light go through the remap
// tables, a removed primitive ends the reuse on the spot (:338-346), and
// ray A is traced against the previous scene (k_di_gen1 queues it under its
// own count for k_trace_prev).
template <class VP>
__device__ void temporal_reuse(const FrameView &F, const ct_params &P, f3 ray_dir, const Shade &S, const Material &mat,
                               Reservoir &res, Reservoir prev, uint32_t prev_index, uint32_t &seed, uint32_t pixel,
                               VP &vp, bool emit_only, RayStats &rs) {
  const bool remap = (F.is_active & CT_REMAP_BIT) != 0;
  prev.M = gmin(prev.M, P.max_influence_from_the_past * res.M);
  const float prev_M = prev.M;
  const float new_M = res.M + prev_M;
  if (res.W_sum > 0.f) {
    float target_lum_at_prev = 0.0f;
    if (luminance(res.F) > 1e-6f) {
      rs.temporal++;
      const ct_di_info &pd = F.prev_di[prev_index];
      Shade ps = shade_from_di(pd);
      if (remap) {
        // get_remapped_primitive_index_by_object_hit (primitives.glsl:133-137)
        const uint32_t gi = F.instances_prev[pd.instance_hit.instance_id].first_primitive_index +
                            pd.instance_hit.primitive_id;
        const uint32_t rp = F.remap_p[gi];
        if (rp == 0xFFFFFFFFu) return;
        if (rp != 0u) ps.prim = rp;
      }
      Material pm = load_material(F, pd.mat_index);
      f3 pro = ld3(pd.ray_origin);
      f3 prd = normalize(ps.P - pro);
      target_lum_at_prev = luminance(reservoir_get_radiance(F, res, prd, ps, pm, pixel, vp, 2u));
    }
    if (emit_only) return;
    const float p_curr = res.M * luminance(res.F);
    const float m_curr = p_curr / gmax(p_curr + prev_M * target_lum_at_prev, 1e-6f);
    res.W_sum *= m_curr;
  }
  if (emit_only) return;
  uint32_t prev_light_index = prev.Y;
  // get_remapped_light_index (primitives.glsl:140-145, :380-387); the
  // re-evaluation below keeps the reservoir's own index, as the shader does
  if (remap && prev.l_type == CT_LIGHT_CUBE && prev_light_index != 0xFFFFFFFFu) {
    const uint32_t t = F.remap_l[prev_light_index];
    if (t != 0u) prev_light_index = t;
  }
  if (prev_light_index != 0xFFFFFFFFu) {
    f3 current_target = reservoir_get_radiance(F, prev, ray_dir, S, mat, pixel, vp, 1u);
    const float target_lum_at_curr = luminance(current_target);
    if (target_lum_at_curr > 0.f) {
      const float target_lum_at_prev = luminance(prev.F);
      const float p_prev = prev.M * target_lum_at_prev;
      const float m_prev = p_prev / gmax(p_prev + res.M * target_lum_at_curr, 1e-6f);
      const float w_prev = m_prev * target_lum_at_curr * prev.W_y;
      update_reservoir(res, prev_light_index, prev.l_type, prev.seed, current_target, w_prev, 1.0f, seed);
    }
  }
  const float target_lum = luminance(res.F);
  res.W_y = target_lum > 0.0f ? res.W_sum / target_lum : 0.0f;
  res.M = new_M;
}
// The previous sample re-evaluated at the current pixel (slot 1): its ray
// does not depend on this frame's visibility, so it is asked for early.
template <class VP>
__device__ void temporal_prev_sample_ray(const FrameView &F, const ct_params &P, f3 ray_dir, const Shade &S,
                                         const Material &mat, const Reservoir &res, Reservoir prev, uint32_t pixel,
                                         VP &vp) {
  prev.M = gmin(prev.M, P.max_influence_from_the_past * res.M);
  if (prev.Y != 0xFFFFFFFFu) reservoir_get_radiance(F, prev, ray_dir, S, mat, pixel, vp, 1u);
}

// stage 0, generate: RIS, then ask for the RIS visibility ray (slot 0) and
// the previous sample's ray (slot 1).  Writes the pre-visibility reservoir to
// RESTIR.intermediate_reservoir and the seed/confidence to the DI record.
// Two instantiations, both launched: each returns at once unless the status
// block's RIS_BRDF_BIT matches, so that the BRDF candidates' closest-hit walk
// never weighs on the registers of the common kernel.
// RIS is latency bound at low occupancy: 12 blocks per SM (40 registers,
// spills) measured 1.45 ms per 1080p frame against 1.55 ms at 10, 1.62 ms
// at 8 (64 registers) and 1.75 ms at 4 (128 registers)
#ifndef CT_GEN0_MIN_BLOCKS
#define CT_GEN0_MIN_BLOCKS 12
#endif
template <bool BRDF>
__global__ void __launch_bounds__(128, BRDF ? 1 : CT_GEN0_MIN_BLOCKS) k_di_gen0(ct_push_constant pc, ct_params P,
                                                                          Workspace ws, DevAccel A) {
  __shared__ BlockConsts B;
  __shared__ int other_variant;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    // the flag first: the instantiation that does not run returns before
    // building the frame view
    const ct_status_block *st = (const ct_status_block *)(uintptr_t)pc.status_buffer;
    other_variant = ((st->is_active & CT_RIS_BRDF_BIT) != 0) != BRDF;
    if (!other_variant) load_frame_view(pc, B);
  }
  __syncthreads();
  if (other_variant) return;  // the same for the whole block
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  const uint32_t screen_pos = y * F.W + x;
  bool active = false;
  f3 d = mk3(0.f);
  Shade S = {};
  Material mat = {};
  Temporal T = {};
  Reservoir res = reservoir_empty();
  bool ris_vis = true;
  if (x < F.W && y < F.H) {
    ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      active = true;
      rs.hits = 1;
      f3 o;
      camera_ray(B, x, y, o, d);
      S = shade_from_di(dref);
      mat = load_material(F, S.mat_index);
      T = gather_temporal(F, P, x, y, screen_pos);
      uint32_t seed = dref.seed;
      res = ris_candidates<BRDF>(F, A, P, o, d, S, mat, T.confidence, seed, screen_pos, ris_vis, rs);
      if constexpr (BRDF) turn_after_ris(F, S, d);
      store_reservoir(F.int_reservoir, screen_pos, res);
      // slot 0 is set every frame: a visibility pass that asks for no ray
      // (no point of the light faces the shading point) leaves no answer
      // there, and a marker left from an earlier frame must not read as SKIP
      ws.vis[screen_pos * CT_VIS_SLOTS] = ris_vis ? 0u : CT_VIS_SKIP;
      dref.seed = seed;
      dref.confidence = T.confidence;
    }
  }
  auto rays = [&](auto &vp) {
    if (!active) return;
    Reservoir tmp = res;
    if (ris_vis) ris_visibility(F, tmp, S, screen_pos, vp);
    if (T.prev.W_y > 0.0f) temporal_prev_sample_ray(F, P, d, S, mat, res, T.prev, screen_pos, vp);
  };
  VisCount cnt{0};
  rays(cnt);
  VisEmit emit{ws.q, screen_pos * CT_VIS_SLOTS, screen_pos, block_reserve(cnt.n, ws.q.count)};
  rays(emit);
  count_rays(P, rs);
}

// queue counter (in the workspace's counter block) of the rays traced against
// the previous scene after an edit
#define CT_PREV_COUNT 4u

// stage 0, second generate: apply the RIS visibility answer, then ask for the
// current sample's ray at the previous pixel (slot 2).  After a scene edit
// (CT_REMAP_BIT) that ray goes to the previous-scene count instead, for
// k_trace_prev.
__global__ void __launch_bounds__(128) k_di_gen1(ct_push_constant pc, ct_params P, Workspace ws) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  const uint32_t screen_pos = y * F.W + x;
  bool active = false;
  f3 d = mk3(0.f);
  Shade S = {};
  Material mat = {};
  Temporal T = {};
  Reservoir res = reservoir_empty();
  uint32_t seed = 0;
  if (x < F.W && y < F.H) {
    const ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      S = shade_from_di(dref);
      if (F.is_active & CT_RIS_BRDF_BIT) {
        f3 o;
        camera_ray(B, x, y, o, d);
        turn_after_ris(F, S, d);
      }
      res = load_reservoir(F.int_reservoir, screen_pos);
      VisRead rd{ws.vis, screen_pos * CT_VIS_SLOTS};
      if (ws.vis[screen_pos * CT_VIS_SLOTS] != CT_VIS_SKIP) {
        ris_visibility(F, res, S, screen_pos, rd);
        store_reservoir(F.int_reservoir, screen_pos, res);
      }
      T = gather_temporal(F, P, x, y, screen_pos);
      if (T.prev.W_y > 0.0f) {
        active = true;
        f3 o;
        camera_ray(B, x, y, o, d);
        mat = load_material(F, S.mat_index);
        seed = dref.seed;
      }
    }
  }
  auto rays = [&](auto &vp, RayStats &st) {
    if (!active) return;
    Reservoir r2 = res;
    uint32_t s2 = seed;
    temporal_reuse(F, P, d, S, mat, r2, T.prev, T.prev_index, s2, screen_pos, vp, true, st);
  };
  if (F.is_active & CT_REMAP_BIT) {  // the same for every thread
    // rays against the previous scene: their own count, walked by k_trace_prev
    VisCount cnt{0};
    RayStats dummy = {};
    rays(cnt, dummy);
    VisEmit emit{ws.q, screen_pos * CT_VIS_SLOTS, screen_pos, block_reserve(cnt.n, ws.q.count + CT_PREV_COUNT)};
    rays(emit, rs);
  } else {
    VisCount cnt{0};
    RayStats dummy = {};
    rays(cnt, dummy);
    VisEmit emit{ws.q, screen_pos * CT_VIS_SLOTS, screen_pos, block_reserve(cnt.n, ws.q.count)};
    rays(emit, rs);
  }
  count_rays(P, rs);
}

// stage 0, resolve: temporal reuse with both answers; final intermediate
// reservoir and DI seed.
// 8 blocks of 128 per SM (64 registers): 0.28 ms per 1080p frame against
// 0.35 ms with the register count left free
#ifndef CT_DI_RESOLVE0_MIN_BLOCKS
#define CT_DI_RESOLVE0_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(128, CT_DI_RESOLVE0_MIN_BLOCKS) k_di_resolve0(ct_push_constant pc, ct_params P, Workspace ws) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  if (x < F.W && y < F.H) {
    const uint32_t screen_pos = y * F.W + x;
    ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      const Temporal T = gather_temporal(F, P, x, y, screen_pos);
      if (T.prev.W_y > 0.0f) {
        f3 o, d;
        camera_ray(B, x, y, o, d);
        Shade S = shade_from_di(dref);
        turn_after_ris(F, S, d);
        const Material mat = load_material(F, S.mat_index);
        Reservoir res = load_reservoir(F.int_reservoir, screen_pos);
        VisRead rd{ws.vis, screen_pos * CT_VIS_SLOTS};
        uint32_t seed = dref.seed;
        RayStats dummy = {};
        temporal_reuse(F, P, d, S, mat, res, T.prev, T.prev_index, seed, screen_pos, rd, false, dummy);
        store_reservoir(F.int_reservoir, screen_pos, res);
        dref.seed = seed;
      }
    }
  }
  count_rays(P, rs);
}

// ---------------------------------------------------------------------------
// SPATIAL_REUSE with defensive pairwise MIS (restir_resampling.glsl:418-540,
// pairwise_mis.glsl:15-114), in three passes per round:
//   select  (per pixel)            neighbour choice, which consumes the
//                                   pixel's random numbers;
//   sample  (per pixel and sample)  each of the two re-evaluations per
//                                   neighbour: neighbour i's sample at this
//                                   pixel (slot 2i) and this pixel's sample at
//                                   neighbour i (slot 2i+1); stores the
//                                   radiance it would have if visible and
//                                   queues its shadow ray;
//   resolve (per pixel)            pairwise MIS with the answers.

// neighbour choice (restir_resampling.glsl:425-500)
__device__ uint32_t spatial_select(const FrameView &F, const ct_params &P, float res_W_y, float confidence, uint32_t cx,
                                   uint32_t cy, float distance, uint32_t &seed, uint32_t *idx) {
  if (res_W_y == 0.f) confidence = 0.0f;
  uint32_t n = 0;
  const float radius = gmix(P.max_neighbors_radius, P.min_neighbors_radius,
                            gclamp(distance / P.max_distance_to_hit, 0.0f, 1.0f));
  uint32_t count = f2u(gmix((float)P.max_num_of_neighbors, (float)P.min_num_of_neighbors, gclamp(confidence, 0.0f, 1.0f)));
  if (count > CT_MAX_NEIGHBORS) count = CT_MAX_NEIGHBORS;
  for (uint32_t i = 0; i < count; i++) {
    float r0 = rnd(seed);
    float r1 = rnd(seed);
    f2 off = 2.0f * f2{r0, r1} - 1.0f;
    off.x = (float)(cx + (uint32_t)f2i(off.x * radius));
    off.y = (float)(cy + (uint32_t)f2i(off.y * radius));
    if (off.x < 0.f || off.x >= (float)F.W || off.y < 0.f || off.y >= (float)F.H) continue;
    if (off.x == (float)cx && off.y == (float)cy) continue;
    const uint32_t ux = f2u(off.x), uy = f2u(off.y);
    const uint32_t lin = uy * F.W + ux;
    if (F.di[lin].distance <= 0.f) continue;
    idx[n++] = lin;
  }
  return n;
}

__global__ void __launch_bounds__(128) k_spatial_select(ct_push_constant pc, ct_params P, Workspace ws, int src_sel) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  const ct_reservoir *src = src_sel ? F.cur_reservoir : F.int_reservoir;
  uint32_t x, y;
  pixel_of(x, y);
  if (x >= F.W || y >= F.H) return;
  const uint32_t screen_pos = y * F.W + x;
  const ct_di_info &dref = F.di[screen_pos];
  uint32_t n = 0, seed = dref.seed;
  if (dref.distance > 0.0f) {
    uint32_t idx[CT_MAX_NEIGHBORS];
    n = spatial_select(F, P, src[screen_pos].W_y, dref.confidence, x, y, dref.distance, seed, idx);
    for (uint32_t i = 0; i < n; i++) ws.nbr[screen_pos * CT_MAX_NEIGHBORS + i] = idx[i];
  }
  ws.smeta[screen_pos] = make_uint2(n, seed);
}

// Captures the one shadow ray a call site would trace.
struct VisCapture {
  bool traced;
  f3 o, d;
  float dist;
  uint32_t inst, prim;
  bool check;
  __device__ bool operator()(f3 o_, f3 d_, float dist_, uint32_t i_, uint32_t p_, bool c_, uint32_t) {
    traced = true; o = o_; d = d_; dist = dist_; inst = i_; prim = p_; check = c_;
    return true;
  }
};

// one thread per (pixel, sample j < R)
// 48 registers, 1280 threads per SM: 1.43 ms per 1080p frame against 1.50
// ms at 1024, 1.80 ms at 768 and 1.79 ms with the register count left free;
// in blocks of 128 (1.38 ms against 1.43 ms in blocks of 256 and 1.42 ms in
// blocks of 64: fewer threads wait at each block's queue reservation)
#ifndef CT_SPATIAL_SAMPLE_THREADS
#define CT_SPATIAL_SAMPLE_THREADS 128
#endif
#ifndef CT_SPATIAL_SAMPLE_MIN_BLOCKS
#define CT_SPATIAL_SAMPLE_MIN_BLOCKS (5 * 256 / CT_SPATIAL_SAMPLE_THREADS)
#endif
__global__ void __launch_bounds__(CT_SPATIAL_SAMPLE_THREADS, CT_SPATIAL_SAMPLE_MIN_BLOCKS) k_spatial_sample(ct_push_constant pc, ct_params P, Workspace ws, int src_sel,
                                                       uint32_t R) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  const ct_reservoir *src = src_sel ? F.cur_reservoir : F.int_reservoir;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t pixel = t / R, j = t % R;
  VisCapture cap;
  cap.traced = false;
  f3 rad = mk3(0.f);
  bool active = false;
  if (pixel < F.W * F.H) {
    const uint2 meta = ws.smeta[pixel];
    const uint32_t i = j >> 1;
    if (i < meta.x) {
      active = true;
      const uint32_t nb = ws.nbr[pixel * CT_MAX_NEIGHBORS + i];
      // even j: the neighbour's sample re-evaluated at this pixel; odd j: this
      // pixel's sample re-evaluated at the neighbour.  Both run the same code
      // on per-lane operands, so a warp's lanes stay together.
      const bool own = (j & 1u) != 0u;
      const Reservoir r = load_reservoir(src, own ? pixel : nb);
      if (reservoir_valid(r)) {
        const ct_di_info &d = F.di[own ? nb : pixel];
        const Shade S = shade_from_di(d);
        // the view direction at this pixel is pass 2's camera ray
        // (rgen.glsl:353-354); at the neighbour it points at the offset
        // shading point (restir_resampling.glsl:522-529)
        const f3 from = own ? S.P : ld3(d.position);
        const f3 rd = normalize(from - ld3(d.ray_origin));
        const Material mat = load_material(F, d.mat_index);
        rad = reservoir_get_radiance(F, r, rd, S, mat, pixel, cap, 0u);
      }
    }
  }
  const uint32_t pos = block_reserve(cap.traced ? 1u : 0u, ws.q.count);
  if (active) {
    const uint32_t slot = pixel * CT_VIS_SLOTS + j;
    st3(&ws.rad[3u * slot], rad);
    if (cap.traced) {
      if (pos >= ws.q.capacity) {
        ct_latch_error(CT_ERR_CAPACITY, 5, pixel);
        ws.vis[slot] = 0;
      } else {
        ws.q.a[pos] = make_float4(cap.o.x, cap.o.y, cap.o.z, cap.dist);
        ws.q.b[pos] = make_float4(cap.d.x, cap.d.y, cap.d.z, __uint_as_float(slot));
        ws.q.c[pos] = make_uint2(cap.inst | (cap.check ? 0x80000000u : 0u), cap.prim);
      }
    } else {
      ws.vis[slot] = 0;
    }
  }
}

// stage 1, resolve: pairwise MIS with the stored re-evaluations; the last
// round shades (rgen.glsl:405-509).
__global__ void __launch_bounds__(128) k_spatial_resolve(ct_push_constant pc, ct_params P, Workspace ws, int src_sel,
                                                        int final_pass, int dst_sel) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  const ct_reservoir *src = src_sel ? F.cur_reservoir : F.int_reservoir;
  ct_reservoir *dst = dst_sel ? F.cur_reservoir : F.int_reservoir;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  if (x < F.W && y < F.H) {
    const uint32_t screen_pos = y * F.W + x;
    ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      rs.hits = 1;
      const Material mat = load_material(F, dref.mat_index);
      Reservoir res = load_reservoir(src, screen_pos);
      const uint2 meta = ws.smeta[screen_pos];
      const uint32_t n = meta.x;
      uint32_t seed = meta.y;
      if (n > 0) {
        Reservoir mis = reservoir_empty();
        float m_c = 1.0f;
        float M_s = res.M;
        const uint32_t k = n;
        const bool canon_valid = reservoir_valid(res);
        const uint32_t base = screen_pos * CT_VIS_SLOTS;
        for (uint32_t i = 0; i < n; i++) {
          rs.neighbours++;
          const Reservoir nr = load_reservoir(src, ws.nbr[screen_pos * CT_MAX_NEIGHBORS + i]);
          f3 curr_target = mk3(0.f);
          float m_i = 0.f;
          const bool in_valid = reservoir_valid(nr);
          if (in_valid) {
            if (ws.vis[base + 2u * i]) curr_target = ld3(&ws.rad[3u * (base + 2u * i)]);
            const float p_i_y_i = luminance(nr.F);
            const float p_c_y_i = luminance(curr_target);
            float mi = nr.M * p_i_y_i;
            float den = mi + (res.M / (float)k) * p_c_y_i;
            m_i = den > 0.f ? mi / den : 0.f;
          }
          f3 input_target = mk3(0.f);
          if (canon_valid && ws.vis[base + 2u * i + 1u]) input_target = ld3(&ws.rad[3u * (base + 2u * i + 1u)]);
          {  // pairwise_update_m_c
            const float p_i_y_c = luminance(input_target);
            const float p_c_y_c = luminance(res.F);
            const float num = nr.M * p_i_y_c;
            const bool den = (p_c_y_c + num) > 0.f;
            m_c += 1.0f;
            m_c -= den ? num / (num + (res.M / (float)k) * p_c_y_c) : 0.f;
          }
          if (in_valid) {
            const float w_i = luminance(curr_target) * nr.W_y * m_i;
            update_reservoir(mis, nr.Y, nr.l_type, nr.seed, curr_target, w_i, 1.0f, seed);
          }
          M_s += nr.M;
        }
        // pairwise_end (its seed is a copy, pairwise_mis.glsl:222)
        uint32_t seed_copy = seed;
        const float w_c = luminance(res.F) * res.W_y * m_c;
        update_reservoir(mis, res.Y, res.l_type, res.seed, res.F, w_c, 1.0f, seed_copy);
        mis.M = M_s;
        const float tl = luminance(mis.F);
        mis.W_y = tl > 0.f ? mis.W_sum / (tl * (float)(1u + k)) : 0.f;
        res = mis;
      }
      if (final_pass && (P.flags & CT_PARAM_INDIRECT)) {
        // rgen.glsl:405-455 with INDIRECT_ILLUMINATION_ON: the direct part
        // waits in the output image for the indirect part and the emission,
        // which k_pt_spatial adds; the seed goes on in the DI record
        f3 hv = mk3(0.f);
        hv = hv + res.F * res.W_y;
        F.swapchain[screen_pos] = make_float4(hv.x, hv.y, hv.z, 1.0f);
        store_reservoir(F.prev_reservoir, screen_pos, res);
        ct_di_info out = dref;
        out.seed = seed;
        F.prev_di[screen_pos] = out;
      } else if (final_pass) {
        f3 hv = mk3(0.f);
        hv = hv + res.F * res.W_y;
        hv = hv + mat.emission;
        if (isinf(hv.x) || isnan(hv.x)) hv.x = 0.0f;
        if (isinf(hv.y) || isnan(hv.y)) hv.y = 0.0f;
        if (isinf(hv.z) || isnan(hv.z)) hv.z = 0.0f;
        float4 px = make_float4(hv.x, hv.y, hv.z, 1.0f);
        F.swapchain[screen_pos] = px;
        if (F.is_active & CT_TAA_BIT) F.taa_frame[screen_pos] = px;
        store_reservoir(F.prev_reservoir, screen_pos, res);
        ct_di_info out = dref;
        out.seed = seed;
        F.prev_di[screen_pos] = out;
      } else {
        store_reservoir(dst, screen_pos, res);
        dref.seed = seed;
      }
    } else if (final_pass) {
      F.prev_di[screen_pos].distance = 0.0f;
    }
  }
  count_rays(P, rs);
}

// ---------------------------------------------------------------------------
// Shadow rays of the queue.  Persistent warps in rounds of three phases:
//   refill: lanes without a ray take the next rays of the queue (one atomic
//           per warp), set up the walk and store the ray in shared memory;
//   step:   every lane with a walk leaves up to CT_WALK_BUDGET boxes of its
//           ray (shadow_step), queueing a job per dilated cell with a test to
//           make, until the warp's job queue holds 32 jobs or no walk
//           continues;
//   test:   the warp tests the queued jobs, one per lane, and marks the rays
//           they block.
// A ray is answered once it is blocked or its walk has ended with none of its
// jobs blocking.  Writes one byte per ray (1 = visible) at the ray's slot.
// Boxes per round: 8 (5.07 ms per 1080p frame against 5.18 ms at 12 and
// 5.32 ms at 16).
#ifndef CT_WALK_BUDGET
#define CT_WALK_BUDGET 8
#endif
// blocks of 256 per SM the register budget is sized for (64 registers; at
// five blocks, 48 registers, the spills cost more than the occupancy gains)
#ifndef CT_SHADOW_MIN_BLOCKS
#define CT_SHADOW_MIN_BLOCKS 4
#endif
#define CT_SHADOW_WARPS 8
#define CT_SHADOW_JOBS 64  // a step adds at most 32 jobs to fewer than 32
// COUNT: the work counters of CT_PARAM_COUNT_RAYS, compiled out of the
// instantiation frames run without them
template <bool COUNT>
__global__ void __launch_bounds__(256, CT_SHADOW_MIN_BLOCKS) k_trace_shadow(DevAccel A, ct_params P, Workspace ws) {
  __shared__ ShadowRay s_ray[CT_SHADOW_WARPS][32];
  __shared__ uint4 s_job[CT_SHADOW_WARPS][CT_SHADOW_JOBS];
  __shared__ uint32_t s_blocked[CT_SHADOW_WARPS];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t lanes_below = (1u << lane) - 1u;
  ShadowRay *rays = s_ray[warp];
  uint4 *jobs = s_job[warp];
  const uint32_t n = ws.q.count[0];
  uint32_t *cursor = ws.q.count + 1;
  RayStats rs = {};
  DdaState st;
  float stop = 0.f;         // the walk's fixed stop distance
  int walk = DDA_DONE;      // the lane's walk: DDA_MORE while it continues
  bool active = false;      // the lane holds an unanswered ray
  bool exhausted = false;
  uint32_t slot = 0, qid = 0;
  for (;;) {
    // refill
    const bool need = !active && !exhausted;
    const unsigned needmask = __ballot_sync(0xFFFFFFFFu, need);
    if (needmask) {
      const uint32_t leader = __ffs(needmask) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(cursor, (uint32_t)__popc(needmask));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (need) {
        const uint32_t id = base + __popc(needmask & lanes_below);
        if (id >= n) {
          exhausted = true;
        } else {
          const float4 a = ws.q.a[id];
          const float4 b = ws.q.b[id];
          const uint2 c = ws.q.c[id];
          qid = id;
          slot = __float_as_uint(b.w);
          rs.shadow++;
          ShadowRay &R = rays[lane];
          if (shadow_ray_begin(A, R, st, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, a.w, c.x & 0x7FFFFFFFu, c.y,
                               (c.x & 0x80000000u) != 0)) {
            active = true;
            walk = DDA_MORE;
            stop = fminf(R.tmax, R.target_t);
          } else {
            ws.vis[slot] = 1;  // nothing to walk: visible
          }
        }
      }
    }
    if (!__any_sync(0xFFFFFFFFu, active || !exhausted)) break;
    // step
    uint32_t njobs = 0;
    {
      const DevGrid &g = A.grids[active ? rays[lane].inst : 0];
      for (int it = 0; it < CT_WALK_BUDGET; it++) {
        bool job = false;
        uint4 jb;
        if (walk == DDA_MORE) {
          // the ray from shared memory: the registers it frees buy a fourth
          // block per SM (walker 10.50 ms per 1080p frame against 10.60 ms
          // with the ray in registers at three blocks)
          walk = shadow_step(A, g, rays[lane].r, st, stop, lane, rs, job, jb);
          if (walk == DDA_LIMIT) ct_latch_error(CT_ERR_ITER_LIMIT, 2, slot / CT_VIS_SLOTS);
        }
        const unsigned jm = __ballot_sync(0xFFFFFFFFu, job);
        if (job) jobs[njobs + __popc(jm & lanes_below)] = jb;
        njobs += __popc(jm);
        if (njobs >= 32u || !__any_sync(0xFFFFFFFFu, walk == DDA_MORE)) break;
      }
    }
    // test
    if (lane == 0) s_blocked[warp] = 0u;
    __syncwarp();
    uint32_t tests = 0;
    for (uint32_t j = lane; j < njobs; j += 32u) {
      const uint4 jb = jobs[j];
      const uint32_t owner = shadow_job_lane(jb);
      if (shadow_job_blocked(A, rays[owner], jb, tests)) atomicOr(&s_blocked[warp], 1u << owner);
    }
    rs.voxel_tests += tests;
    __syncwarp();
    // answer
    if (active) {
      if ((s_blocked[warp] >> lane) & 1u) {
        ws.vis[slot] = 0;
        active = false;
        walk = DDA_DONE;
      } else if (walk != DDA_MORE) {
        // the walk of this instance ended unblocked: the next instance, if any
        const float4 a = ws.q.a[qid], b = ws.q.b[qid];
        ShadowRay &R = rays[lane];
        if (R.inst + 1 < A.n_grids &&
            shadow_ray_next(A, R, st, R.inst + 1, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z})) {
          walk = DDA_MORE;
        } else {
          ws.vis[slot] = 1;
          active = false;
        }
      }
    }
    __syncwarp();
  }
  rs.walker_bricks = rs.bricks;
  if constexpr (COUNT) count_rays(P, rs);
}

// The rays k_di_gen1 queued against the previous scene after an edit
// (vertex_visible_prev), one thread per ray; returns at once in the frames
// without an edit, whose previous-scene count is 0.
__global__ void __launch_bounds__(128) k_trace_prev(ct_push_constant pc, DevAccel A_prev, ct_params P, Workspace ws) {
  const uint32_t n = ws.q.count[CT_PREV_COUNT];
  if (n == 0) return;  // the same for every thread
  const ct_world *wd = (const ct_world *)(uintptr_t)pc.world_buffer;
  FrameView F;  // the two tables vertex_visible_prev reads
  F.instances = (const ct_instance *)(uintptr_t)wd->instance_address;
  F.aabbs = (const ct_aabb *)(uintptr_t)wd->aabb_address;
  RayStats rs = {};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i >= ws.q.capacity) break;
    const float4 a = ws.q.a[i], b = ws.q.b[i];
    const uint2 c = ws.q.c[i];
    const uint32_t slot = __float_as_uint(b.w);
    rs.shadow++;
    ws.vis[slot] = vertex_visible_prev(A_prev, F, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, a.w, c.x & 0x7FFFFFFFu, c.y,
                                       (c.x & 0x80000000u) != 0, slot / CT_VIS_SLOTS, rs)
                       ? 1
                       : 0;
  }
  count_rays(P, rs);
}

// ---------------------------------------------------------------------------
// TAA (taa.glsl:16-109); the grid covers (W/8)*8 x (H/8)*8 pixels like the
// reference dispatch.
__global__ void __launch_bounds__(64) k_taa(ct_push_constant pc, ct_params P) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    // only the frame view is needed
    load_frame_view(pc, B);
  }
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  if (x >= F.W || y >= F.H) return;
  const uint32_t idx = x + y * F.W;
  ct_di_info di = F.di[idx];
  if (!(di.distance > 0.0f)) return;
  const f3 n = ld3(di.normal);
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  uint32_t count = 0;
  for (int i = -1; i <= 1; i++) {
    for (int j = -1; j <= 1; j++) {
      int nx = (int)x + i, ny = (int)y + j;
      if ((float)nx < 0.0f || nx >= (int)F.W || (float)ny < 0.0f || ny >= (int)F.H) continue;
      const uint32_t ni = (uint32_t)nx + (uint32_t)ny * F.W;
      const ct_di_info &nd = F.di[ni];
      if (di.distance <= 0.f || di.mat_index != nd.mat_index || (dot(n, ld3(nd.normal)) < 0.906f) ||
          (fabsf(di.distance - nd.distance) > 0.1f * di.distance))
        continue;
      ++count;
      float4 p = F.taa_frame[ni];
      acc.x = acc.x + p.x; acc.y = acc.y + p.y; acc.z = acc.z + p.z; acc.w = acc.w + p.w;
    }
  }
  const float fc = (float)count;
  acc.x = acc.x / fc; acc.y = acc.y / fc; acc.z = acc.z / fc; acc.w = acc.w / fc;
  const ct_velocity vel = F.velocity[idx];
  uint32_t seed = di.seed;
  const float r0 = rnd(seed);
  const float r1 = rnd(seed);
  const f2 xi1 = f2{(float)x, (float)y} + f2{vel.velocity[0], vel.velocity[1]} + f2{r0, r1};
  const int ix = f2i(xi1.x), iy = f2i(xi1.y);
  if (ix >= 0 && ix < (int)F.W && iy >= 0 && iy < (int)F.H) {
    const uint32_t pidx = (uint32_t)ix + (uint32_t)iy * F.W;
    const float4 prev_px = F.previous_swapchain[pidx];
    const ct_di_info &pd = F.prev_di[pidx];
    const bool valid = dot(ld3(pd.normal), n) >= 0.99f && pd.mat_index == di.mat_index;
    if (valid) {
      const float a = P.taa_alpha, b = 1.0f - P.taa_alpha;
      acc.x = a * acc.x + b * prev_px.x;
      acc.y = a * acc.y + b * prev_px.y;
      acc.z = a * acc.z + b * prev_px.z;
      acc.w = a * acc.w + b * prev_px.w;
    }
  }
  F.swapchain[idx] = acc;
}

// ---------------------------------------------------------------------------
// ReSTIR PT
#include "ct_pt.cuh"

// (declared with ris_candidates)
__device__ BrdfCandidates ris_brdf_candidates(const FrameView &F, const DevAccel &A, f3 ray_origin, f3 ray_dir,
                                              Shade S, uint32_t seed, uint32_t nee, uint32_t n_brdf,
                                              uint32_t cube_count, float extent, uint32_t pixel) {
  BrdfCandidates out;
  out.res = reservoir_empty();
  out.moved = false;
  const Material mat = load_material(F, S.mat_index);
  RayStats rs = {};
  f3 P = S.P, n = S.n;
  for (uint32_t l = 0; l < F.light_config.brdf_count; l++) {
    float w_i = 0.0f;
    f3 Fv = mk3(0.f);
    uint32_t light_index = 0xFFFFFFFFu;
    const f3 Pl = P, nl = n;
    const f3 wo = normalize(ray_origin - Pl);
    const uint32_t current_seed = seed;
    f3 wi;
    const bool done = scatter_callable(F, mat.type & 0xFFu, S.mat_index, P, n, ray_dir, seed, pixel, wi);
    const float mat_pdf = sample_material_pdf(mat, n, wo, wi);
    if (P.x != Pl.x || P.y != Pl.y || P.z != Pl.z || n.x != nl.x || n.y != nl.y || n.z != nl.z) out.moved = true;
    if (!done) {
      const Isect i = intersect_closest(F, A, Pl, wi, pixel, rs);
      if (i.is_hit && (i.mat.emission.x > 0.0f || i.mat.emission.y > 0.0f || i.mat.emission.z > 0.0f)) {
        float G = geom_fact_sa(Pl, i.world_hit, i.world_nrm);
        if (isnan(G) || isinf(G) || G < 0.0f) G = 0.0f;
        // sample_lights_pdf (light.glsl:272-291)
        float light_pdf = 1.0f / (float)cube_count;
        light_pdf = light_pdf / (extent * extent * 6.0f);
        const float m_i = 1.f / gmax((float)n_brdf * mat_pdf * G + (float)nee * light_pdf * G, 1e-6f);
        const f3 brdf = evaluate_material(mat, nl, wo, wi);
        Fv = brdf * i.mat.emission * G;
        w_i = luminance(Fv) * m_i;
        light_index = F.primitives[F.instances[i.inst].first_primitive_index + i.prim].light_index;
      }
    }
    update_reservoir(out.res, light_index, CT_LIGHT_CUBE, current_seed, Fv, w_i, 1.0f, seed);
  }
  out.seed = seed;
  return out;
}


__device__ __forceinline__ Isect primary_isect(const FrameView &F, const ct_di_info &d, bool normalized_wo) {
  Isect i;
  i.is_hit = d.distance > 0.0f;
  i.distance = d.distance;
  i.world_hit = ld3(d.position);
  i.world_nrm = ld3(d.normal);
  const f3 wo = ld3(d.ray_origin) - i.world_hit;
  i.wo = normalized_wo ? normalize(wo) : wo;
  i.wi = mk3(0.f);
  i.inst = d.instance_hit.instance_id;
  i.prim = d.instance_hit.primitive_id;
  i.material_idx = d.mat_index;
  i.mat = load_material(F, d.mat_index);
  return i;
}

// temporal_path_reuse (indirect_illumination.glsl:147-281): Talbot RMIS over
// the pixel's new path and the reprojected previous one
// replay_merge / replay_back: the hybrid shift's replays of the temporal
// sample to the current primary hit and of the pixel's new path to the
// previous one
template <bool HYBRID, class VP, class RP>
__device__ PathRes temporal_path_reuse(const FrameView &F, const DevAccel &A, const PtParams &pp, const PathRes &central,
                                       PathRes temporal, uint32_t &seed, const Isect &cur_i, const Isect &prev_i,
                                       VP &vis, const RP &replay_merge, const RP &replay_back) {
  PathRes dst = path_res_init(pp.max_depth);
  const float current_M = central.M;
  temporal.M = gmin(pp.max_influence * current_M, temporal.M);
  float dst_jacobian = 0.f;
  for (int it = -1; it <= 0; ++it) {
    float p_sum = 0.f, p_self = 0.f;
    PathRes temp_dst = dst;
    bool possible = false;
    if (it == -1) {
      temp_dst = central;
      dst_jacobian = 1.f;
      possible = temp_dst.weight > 0.f;
    } else {
      possible =
          shift_and_merge<HYBRID>(F, A, pp, dst_jacobian, cur_i, temp_dst, prev_i, temporal, seed, vis, 1u, replay_merge);
    }
    if (possible) {
      for (int j = -1; j <= 0; ++j) {
        if (j == -1) {
          const float cur_p = path_scalar(temp_dst.F) * current_M;
          p_sum += cur_p;
          if (it == -1) p_self = cur_p;
        } else {
          if (it == j) {
            p_self = path_scalar(temporal.F) / dst_jacobian * temporal.M;
            p_sum += p_self;
            continue;
          }
          float t_jac = 0.f;
          PathRes shifted = temp_dst;
          const f3 integ =
              shift_path<HYBRID>(F, A, pp, t_jac, prev_i, cur_i, shifted, true, vis, it == -1 ? 0u : 2u, replay_back);
          const float p_ = path_scalar(integ) * t_jac;
          p_sum += p_ * temporal.M;
        }
      }
    }
    const float mis_weight = p_sum == 0.f ? 0.f : p_self / p_sum;
    path_res_merge_mis(dst, temp_dst.F, dst_jacobian, temp_dst, seed, mis_weight);
  }
  if (dst.weight > 0.f) path_res_finalize_gris(dst);
  if (dst.weight < 0.f || isinf(dst.weight) || isnan(dst.weight)) dst.weight = 0.f;
  return dst;
}

// Scratch of the path wavefront (ct_workspace_size with CT_PARAM_INDIRECT):
// one PathState per pixel, the closest hit of each pixel's current bounce
// ray, and two ray queues (origin + pixel, direction) used in turn; queue
// counts and walker cursors live in the workspace's counter block.
// The hybrid shift's replays of temporal reuse, per pixel two slots (the
// temporal sample shifted to the current primary hit, the new path shifted
// to the previous one): hit.w the state (0 failed, 1 done, 2 not asked for,
// 3 asked for), the replay's last vertex (hit point, normal, wo, material,
// instance, primitive) and the prefix throughput.
struct __align__(16) ReplayOut {
  float4 hit;  // xyz world hit, w state
  float4 nrm;  // xyz world normal, w material index bits
  float4 wo;   // xyz wo, w instance bits
  float4 tp;   // xyz prefix throughput, w primitive bits
};
#define CT_REPLAY_FAILED 0u
#define CT_REPLAY_DONE 1u
#define CT_REPLAY_NOT_ASKED 2u
#define CT_REPLAY_ASKED 3u
// Path states in 16-byte columns: column c of path i is col[c * n + i], so
// that a warp's accesses to one column are 512 contiguous bytes (the
// array-of-structs layout had every lane's 16-byte access in its own 256 B
// record).  Kernels hold a PathState in registers and move whole columns.
constexpr uint32_t kPathCols = (uint32_t)((sizeof(PathState) + 15) / 16);
union PathCols {
  PathState p;
  uint4 u[kPathCols];
};
struct PathStore {
  uint4 *col;
  uint32_t n;  // paths (pixels)
  // the columns whose bit is set in MASK; the fields in the others are left unset
  template <uint32_t MASK = 0xFFFFFFFFu>
  __device__ __forceinline__ PathState load(uint32_t i) const {
    PathCols v;
#pragma unroll
    for (uint32_t c = 0; c < kPathCols; c++)
      if ((MASK >> c) & 1u) v.u[c] = col[(size_t)c * n + i];
    return v.p;
  }
  __device__ __forceinline__ void store(uint32_t i, const PathState &p) const {
    PathCols v;
    v.p = p;
#pragma unroll
    for (uint32_t c = 0; c < kPathCols; c++) col[(size_t)c * n + i] = v.u[c];
  }
};
// the columns a bit mask of fields [offset, offset + size) spans
__host__ __device__ constexpr uint32_t path_cols(size_t offset, size_t size) {
  uint32_t m = 0;
  for (size_t c = offset / 16; c <= (offset + size - 1) / 16; c++) m |= 1u << c;
  return m;
}
struct PtWork {
  PathStore state;
  uint4 *hit;      // per pixel: instance (0xFFFFFFFF: miss), primitive, global primitive
  float4 *q[2];    // 2 float4 per entry
  uint32_t *count; // [0] q0 count, [1] q0 cursor, [2] q1 count, [3] q1 cursor, [4] replay jobs
  uint32_t capacity;
  ReplayOut *replay;  // hybrid shift only: 2 per pixel
  uint32_t *jobs;     // hybrid shift only: 2 per pixel, pixel * 2 + slot
};
static_assert(kPathCols * 16 <= CT_PT_STATE_BYTES, "PathState outgrew its workspace slot");

// pass 1, ReSTIR PT block, part 1: the path starts at the primary hit; its
// first bounce ray goes to queue 0
__global__ void __launch_bounds__(128) k_pt_start(ct_push_constant pc, DevAccel A, ct_params P, PtWork w) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  bool emit = false;
  uint32_t screen_pos = 0;
  PathState path;
  if (x < F.W && y < F.H) {
    screen_pos = y * F.W + x;
    const ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      const PtParams pp = pt_params(F, P, A);
      if (pp.max_depth >= CT_PT_MAX_ITER) ct_latch_error(CT_ERR_UNSUPPORTED, 6, screen_pos);
      f3 o, d;
      camera_ray(B, x, y, o, d);
      const Isect cur_i = primary_isect(F, dref, true);
      emit = path_start(F, pp, path, o, d, cur_i, dref.seed, screen_pos);
      if (!emit) path_finish(path);
      w.state.store(screen_pos, path);
    }
  }
  const uint32_t pos = block_reserve(emit ? 1u : 0u, w.count);
  if (emit) {
    if (pos >= w.capacity) {
      ct_latch_error(CT_ERR_CAPACITY, 7, screen_pos);
    } else {
      w.q[0][2u * pos] = make_float4(path.origin.x, path.origin.y, path.origin.z, __uint_as_float(screen_pos));
      w.q[0][2u * pos + 1u] = make_float4(path.dir.x, path.dir.y, path.dir.z, 0.f);
    }
  }
}

// closest hits of the bounce rays in queue `qi`: persistent lanes, each
// walks one ray a bounded number of cells per turn and takes the next ray of
// the queue when its ray is done (one atomic per warp refill)
#ifndef CT_EXTEND_MIN_BLOCKS
#define CT_EXTEND_MIN_BLOCKS 3
#endif
// boxes per turn: 4 (1.04-1.05 ms per 1080p frame against 1.06-1.07 ms at
// 6, 1.10 ms at 8 and 1.15 ms at 12)
#ifndef CT_EXTEND_BUDGET
#define CT_EXTEND_BUDGET 4
#endif
template <bool COUNT>
__global__ void __launch_bounds__(256, CT_EXTEND_MIN_BLOCKS) k_pt_extend(DevAccel A, ct_params P, PtWork w, int qi) {
  const uint32_t n = w.count[2 * qi];
  uint32_t *cursor = w.count + 2 * qi + 1;
  const float4 *q = w.q[qi];
  const uint32_t lane = threadIdx.x & 31u;
  __shared__ ObjRay s_ray[256];
  ObjRay &R = s_ray[threadIdx.x];
  RayStats rs = {};
  ClosestWalk cw;
  uint32_t pixel = 0, qid = 0;
  bool active = false, exhausted = false;
  // the lane's bounce ray, read again from the queue when its walk changes instance
  const auto ray = [&](f3 &o, f3 &d) {
    const float4 a = q[2u * qid], b = q[2u * qid + 1u];
    o = f3{a.x, a.y, a.z};
    d = f3{b.x, b.y, b.z};
  };
  for (;;) {
    const bool need = !active && !exhausted;
    const uint32_t needmask = __ballot_sync(0xFFFFFFFFu, need);
    if (needmask) {
      uint32_t base = 0;
      if (lane == (uint32_t)(__ffs(needmask) - 1)) base = atomicAdd(cursor, (uint32_t)__popc(needmask));
      base = __shfl_sync(0xFFFFFFFFu, base, __ffs(needmask) - 1);
      if (need) {
        const uint32_t id = base + (uint32_t)__popc(needmask & ((1u << lane) - 1u));
        if (id >= n) {
          exhausted = true;
        } else {
          const float4 a = q[2u * id], b = q[2u * id + 1u];
          qid = id;
          pixel = __float_as_uint(a.w);
          rs.bounce++;
          if (closest_walk_begin(A, cw, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, R)) {
            w.hit[pixel] = make_uint4(0xFFFFFFFFu, 0u, 0u, 0u);
          } else {
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xFFFFFFFFu, active || !exhausted)) break;
    if (active && closest_walk_advance(A, cw, CT_EXTEND_BUDGET, pixel, rs, ray, R) == DDA_DONE) {
      if (cw.best.hit) rs.bounce_hits++;
      w.hit[pixel] = cw.best.hit ? make_uint4(cw.best.inst, cw.best.prim, cw.best.gprim, 0u)
                                 : make_uint4(0xFFFFFFFFu, 0u, 0u, 0u);
      active = false;
    }
  }
  if constexpr (COUNT) count_rays(P, rs);
}

// shades the vertices the rays of queue `qi` found; paths that go on put
// their next bounce ray in the other queue, light samples put their shadow
// ray in the shadow-ray queue
// 2 blocks of 256 per SM (128 registers): 0.90 ms per 1080p frame against
// 1.08 ms at 1 block (212 registers), with the path states in columns
#ifndef CT_SHADE_MIN_BLOCKS
#define CT_SHADE_MIN_BLOCKS 2
#endif
__global__ void __launch_bounds__(256, CT_SHADE_MIN_BLOCKS) k_pt_shade(ct_push_constant pc, DevAccel A, ct_params P, Workspace ws,
                                                  PtWork w, int qi) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  const PtParams pp = pt_params(F, P, A);
  const uint32_t n = w.count[2 * qi];
  const int qo = qi ^ 1;
  RayStats rs = {};
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t id = base + threadIdx.x;
    bool next = false;
    uint32_t pixel = 0;
    VisRecord nee{false};
    PathState path;
    if (id < n) {
      pixel = __float_as_uint(w.q[qi][2u * id].w);
      path = w.state.load(pixel);
      const uint4 h = w.hit[pixel];
      path_shade(F, A, pp, path, h.x != 0xFFFFFFFFu, h.x, h.y, h.z, nee, pixel);
      next = path_active(path);
      if (!next) path_finish(path);
      w.state.store(pixel, path);
    }
    const uint32_t pos = block_reserve(next ? 1u : 0u, w.count + 2 * qo);
    if (next) {
      if (pos >= w.capacity) {
        ct_latch_error(CT_ERR_CAPACITY, 7, pixel);
      } else {
        w.q[qo][2u * pos] = make_float4(path.origin.x, path.origin.y, path.origin.z, __uint_as_float(pixel));
        w.q[qo][2u * pos + 1u] = make_float4(path.dir.x, path.dir.y, path.dir.z, 0.f);
      }
    }
    const uint32_t npos = block_reserve(nee.has ? 1u : 0u, ws.q.count);
    if (nee.has) {
      if (npos >= ws.q.capacity) {
        ct_latch_error(CT_ERR_CAPACITY, 8, pixel);
      } else {
        ws.q.a[npos] = nee.a;
        ws.q.b[npos] = make_float4(nee.b.x, nee.b.y, nee.b.z, __uint_as_float(pixel * CT_VIS_SLOTS + (CT_VIS_SLOTS - 1u)));
        ws.q.c[npos] = nee.c;
      }
    }
  }
  count_rays(P, rs);
}

// The paths still running after CT_PT_TAIL_ROUND wavefront rounds are few,
// and each later round would wait for its slowest walk: one thread per path
// finishes them here, walking each bounce ray in place and shading its
// vertex, for the remaining rounds of the CT_PT_MAX_ITER bound.  Light-sample
// rays go to the shadow-ray queue while it has room (their answers are not
// read) and are walked in place otherwise.  With 8 wavefront rounds, paths
// of up to 8 bounces never get here and the launch replaces the empty
// rounds; earlier switches were measured slower on the 1080p terrain (one
// thread per path walks and shades much slower per path than the wavefront).
#ifndef CT_PT_TAIL_ROUND
#define CT_PT_TAIL_ROUND 8
#endif
__global__ void __launch_bounds__(128) k_pt_finish(ct_push_constant pc, DevAccel A, ct_params P, Workspace ws,
                                                   PtWork w, int qi) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  const PtParams pp = pt_params(F, P, A);
  const uint32_t n = w.count[2 * qi];
  RayStats rs = {};
  for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    const uint32_t pixel = __float_as_uint(w.q[qi][2u * id].w);
    PathState path = w.state.load(pixel);
    for (int round = CT_PT_TAIL_ROUND; round < CT_PT_MAX_ITER; round++) {
      rs.bounce++;
      ClosestWalk cw;
      NoObjRay R;
      const auto ray = [&](f3 &o, f3 &d) { o = path.origin; d = path.dir; };
      if (!closest_walk_begin(A, cw, path.origin, path.dir, R))
        while (closest_walk_advance(A, cw, 1 << 20, pixel, rs, ray, R) == DDA_MORE) {
        }
      if (cw.best.hit) rs.bounce_hits++;
      VisRecord nee{false};
      path_shade(F, A, pp, path, cw.best.hit, cw.best.inst, cw.best.prim, cw.best.gprim, nee, pixel);
      if (nee.has) {
        const uint32_t pos = atomicAdd(ws.q.count, 1u);
        if (pos < ws.q.capacity) {
          ws.q.a[pos] = nee.a;
          ws.q.b[pos] = make_float4(nee.b.x, nee.b.y, nee.b.z, __uint_as_float(pixel * CT_VIS_SLOTS + (CT_VIS_SLOTS - 1u)));
          ws.q.c[pos] = nee.c;
        } else {
          rs.shadow++;
          vertex_visible(A, f3{nee.a.x, nee.a.y, nee.a.z}, f3{nee.b.x, nee.b.y, nee.b.z}, nee.a.w,
                         nee.c.x & 0x7FFFFFFFu, nee.c.y, (nee.c.x & 0x80000000u) != 0, pixel, rs);
        }
      }
      if (!path_active(path)) {
        path_finish(path);
        break;
      }
    }
    w.state.store(pixel, path);
  }
  count_rays(P, rs);
}

// Visibility of temporal path reuse: call sites 0 (new path seen from the
// previous primary hit) and 1 (previous path at the new primary hit) do not
// depend on any answer and are queued by the first pass; call site 2
// (previous path seen from the previous primary hit) runs only when site 1's
// shift was selected, and the second pass traces it in place.  Answers live
// in the pixel's visibility slots CT_PT_TEMPORAL_SLOT + site.
#define CT_PT_TEMPORAL_SLOT 12u
struct VisPT {
  const uint8_t *ans;
  uint32_t base;       // pixel * CT_VIS_SLOTS + CT_PT_TEMPORAL_SLOT
  uint32_t emit_mask;  // call sites whose ray is recorded (answered "visible")
  uint32_t read_mask;  // call sites whose answer is read
  uint32_t n;
  float4 a[2], b[2];
  uint2 c[2];
  __device__ bool operator()(f3 o, f3 d, float dist, uint32_t inst, uint32_t prim, bool check, uint32_t site) {
    if ((read_mask >> site) & 1u) return ans[base + site] != 0;
    if (((emit_mask >> site) & 1u) && dist >= 0.0f && n < 2u) {
      a[n] = make_float4(o.x, o.y, o.z, dist);
      b[n] = make_float4(d.x, d.y, d.z, __uint_as_float(base + site));
      c[n] = make_uint2(inst | (check ? 0x80000000u : 0u), prim);
      n++;
    }
    return true;
  }
};

// The final temporal pass: the answers of call sites 0 and 1 come from the
// queue walked after PHASE 0; site 2 (the temporal sample shifted back, rare
// because it follows a successful shift) is traced in place.  A ray with an
// empty range [0, distance] is visible, as the shader's query is.
struct VisPTFinal {
  const uint8_t *ans;
  uint32_t base;
  const DevAccel &A;
  uint32_t pixel;
  RayStats &rs;
  __device__ bool operator()(f3 o, f3 d, float dist, uint32_t inst, uint32_t prim, bool check, uint32_t site) {
    if (site < 2u) return ans[base + site] != 0;
    if (!(dist >= 0.0f)) return true;
    rs.shadow++;
    return vertex_visible(A, o, d, dist, inst, prim, check, pixel, rs);
  }
};

// The inputs of temporal path reuse for one hit pixel: the new path's
// reservoir, the reprojected previous one (temporal_path_get_reprojected,
// indirect_illumination.glsl:30-59, which draws two numbers from the
// pixel's seed), and the two primary hits.
struct TemporalSetup {
  PathRes central, temporal;
  Isect cur_i, prev_i;
  uint32_t seed;
  bool overflow;  // the path had more bounces than the wavefront ran
};
__device__ __forceinline__ TemporalSetup temporal_setup(const FrameView &F, const PtWork &w, uint32_t x, uint32_t y,
                                                        uint32_t screen_pos, const ct_di_info &dref) {
  TemporalSetup t;
  // only the columns of the fields read here
  constexpr uint32_t kCols = path_cols(offsetof(PathState, flags), sizeof(uint32_t)) |
                             path_cols(offsetof(PathState, seed), sizeof(uint32_t)) |
                             path_cols(offsetof(PathState, res), sizeof(PathRes));
  const PathState ps = w.state.load<kCols>(screen_pos);
  t.central = ps.res;
  t.seed = ps.seed;
  t.overflow = (ps.flags & CT_PF_ACTIVE) != 0;
  if (t.overflow) {
    t.central.M = 1.0f;
    path_res_finalize_ris(t.central);
  }
  t.cur_i = primary_isect(F, dref, true);
  const ct_velocity vel = F.velocity[screen_pos];
  f2 xi1 = f2{(float)x, (float)y} + f2{vel.velocity[0], vel.velocity[1]};
  const float r1 = rnd(t.seed);
  const float r2 = rnd(t.seed);
  xi1 = xi1 + f2{r1, r2};
  uint32_t prev_idx = f2u(xi1.x) + f2u(xi1.y) * F.W;
  prev_idx = gmin(F.W * F.H - 1u, prev_idx);
  t.temporal = load_path_res(F.temporal_path_reservoir[prev_idx]);
  t.prev_i = primary_isect(F, F.prev_di[prev_idx], false);
  return t;
}

// shift_hybrid would replay `src` (the conditions it checks before replaying)
__device__ __forceinline__ bool needs_replay(const PathRes &src) {
  const uint32_t rc_length = pf_rc_length(src.path_flags), path_length = pf_path_length(src.path_flags);
  return src.weight != 0.f && rc_length > 1u && (rc_length <= path_length || path_length + 1u == rc_length) &&
         objhit_exists(src.rc_hit.inst, src.rc_hit.prim);
}

// Hybrid shift, before temporal reuse: every hit pixel lists the replays its
// temporal reuse will ask for (slot 0 with the temporal sample, slot 1 with
// the new path, which is shifted only when its weight is positive) and
// marks the others as not asked for.
__global__ void __launch_bounds__(128) k_pt_replay_jobs(ct_push_constant pc, PtWork w) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  bool want[2] = {false, false};
  uint32_t screen_pos = 0;
  if (x < F.W && y < F.H) {
    screen_pos = y * F.W + x;
    const ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      const TemporalSetup t = temporal_setup(F, w, x, y, screen_pos, dref);
      want[0] = needs_replay(t.temporal);
      want[1] = t.central.weight > 0.f && needs_replay(t.central);
    }
    for (int k = 0; k < 2; k++)
      w.replay[2u * screen_pos + k].hit.w = __uint_as_float(want[k] ? CT_REPLAY_ASKED : CT_REPLAY_NOT_ASKED);
  }
  for (int k = 0; k < 2; k++) {
    const uint32_t pos = block_reserve(want[k] ? 1u : 0u, w.count + 4);
    if (want[k]) w.jobs[pos] = 2u * screen_pos + (uint32_t)k;
    __syncthreads();  // block_reserve's shared scratch is read before the next call writes it
  }
}

// Hybrid shift: the replays the jobs list, one per thread over a grid
// stride, so that a warp walks 32 replays side by side instead of waiting
// on one lane of a pixel kernel.
__global__ void __launch_bounds__(128) k_pt_replay(ct_push_constant pc, DevAccel A, ct_params P, PtWork w) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  const uint32_t n = w.count[4];
  RayStats rs = {};
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t job = w.jobs[j];
    const uint32_t screen_pos = job >> 1, slot = job & 1u;
    const uint32_t x = screen_pos % F.W, y = screen_pos / F.W;
    const PtParams pp = pt_params(F, P, A);
    const TemporalSetup t = temporal_setup(F, w, x, y, screen_pos, F.di[screen_pos]);
    const Isect &dst = slot == 0u ? t.cur_i : t.prev_i;
    const PathRes &src = slot == 0u ? t.temporal : t.central;
    Isect prev;
    f3 tp = mk3(0.f);
    const bool ok = replay_prefix(F, A, pp, dst, src, pf_rc_length(src.path_flags), prev, tp, screen_pos, rs);
    ReplayOut r;
    r.hit = make_float4(prev.world_hit.x, prev.world_hit.y, prev.world_hit.z,
                        __uint_as_float(ok ? CT_REPLAY_DONE : CT_REPLAY_FAILED));
    r.nrm = make_float4(prev.world_nrm.x, prev.world_nrm.y, prev.world_nrm.z, __uint_as_float(prev.material_idx));
    r.wo = make_float4(prev.wo.x, prev.wo.y, prev.wo.z, __uint_as_float(prev.inst));
    r.tp = make_float4(tp.x, tp.y, tp.z, __uint_as_float(prev.prim));
    if (!ok) r.hit.x = r.hit.y = r.hit.z = 0.f;
    w.replay[2u * screen_pos + slot] = r;
  }
  count_rays(P, rs);
}

// replays k_pt_replay left in a pixel's slot
struct StoredReplay {
  const FrameView &F;
  const ReplayOut *slot;
  uint32_t pixel;
  __device__ bool operator()(const Isect &, const PathRes &, uint32_t, Isect &prev, f3 &tp) const {
    const ReplayOut r = *slot;
    const uint32_t state = __float_as_uint(r.hit.w);
    if (state != CT_REPLAY_DONE) {
      if (state != CT_REPLAY_FAILED) ct_latch_error(CT_ERR_UNSUPPORTED, 44, pixel);  // a replay nobody listed
      return false;
    }
    prev.is_hit = true;
    prev.distance = 0.f;
    prev.world_hit = f3{r.hit.x, r.hit.y, r.hit.z};
    prev.world_nrm = f3{r.nrm.x, r.nrm.y, r.nrm.z};
    prev.wo = f3{r.wo.x, r.wo.y, r.wo.z};
    prev.wi = mk3(0.f);
    prev.inst = __float_as_uint(r.wo.w);
    prev.prim = __float_as_uint(r.tp.w);
    prev.material_idx = __float_as_uint(r.nrm.w);
    prev.mat = load_material(F, prev.material_idx);
    tp = f3{r.tp.x, r.tp.y, r.tp.z};
    return true;
  }
};

// pass 1, ReSTIR PT block, part 2: temporal path reuse of the finished path
// (indirect_illumination.glsl:283-305), indirect colour, DI seed.  PHASE 0
// queues the visibility rays of call sites {0, 1}; PHASE 1 reads their
// answers, traces site 2 in place and writes the results.
template <int PHASE, bool HYBRID>
// both temporal passes at 4 blocks of 128 per SM (128 registers): 1.27 ms
// per 1080p frame against 1.46 ms at 3 blocks / free (pass 1 had 250
// registers) and 1.34 ms at 5 blocks
#ifndef CT_PT_TEMPORAL0_MIN_BLOCKS
#define CT_PT_TEMPORAL0_MIN_BLOCKS 4
#endif
#ifndef CT_PT_TEMPORAL1_MIN_BLOCKS
#define CT_PT_TEMPORAL1_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(128, PHASE == 0 ? CT_PT_TEMPORAL0_MIN_BLOCKS : CT_PT_TEMPORAL1_MIN_BLOCKS) k_pt_temporal(ct_push_constant pc, DevAccel A, ct_params P, Workspace ws,
                                                     PtWork w) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  VisPT vis{ws.vis, 0u, 3u, 0u, 0u};
  uint32_t screen_pos = 0;
  if (x < F.W && y < F.H) {
    screen_pos = y * F.W + x;
    ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      const PtParams pp = pt_params(F, P, A);
      TemporalSetup t = temporal_setup(F, w, x, y, screen_pos, dref);
      if (t.overflow && PHASE == 1) ct_latch_error(CT_ERR_ITER_LIMIT, 6, screen_pos);
      uint32_t &seed = t.seed;
      vis.base = screen_pos * CT_VIS_SLOTS + CT_PT_TEMPORAL_SLOT;
      const StoredReplay replay_merge{F, HYBRID ? w.replay + 2u * screen_pos : nullptr, screen_pos};
      const StoredReplay replay_back{F, HYBRID ? w.replay + 2u * screen_pos + 1u : nullptr, screen_pos};
      if constexpr (PHASE == 0) {
        temporal_path_reuse<HYBRID>(F, A, pp, t.central, t.temporal, seed, t.cur_i, t.prev_i, vis, replay_merge,
                                    replay_back);
      } else {
        VisPTFinal fin{ws.vis, vis.base, A, screen_pos, rs};
        const PathRes res = temporal_path_reuse<HYBRID>(F, A, pp, t.central, t.temporal, seed, t.cur_i, t.prev_i, fin,
                                                        replay_merge, replay_back);
        rs.hits = 1;
        rs.temporal = 1;
        store_path_res(F.out_path_reservoir[screen_pos], res);
        f3 ind = res.F * res.weight;
        if (any_nan_inf(ind)) ind = mk3(0.f);
        st3(F.indirect_color + 3u * screen_pos, ind);
        dref.seed = seed;
      }
    }
  }
  if constexpr (PHASE == 0) {
    const uint32_t pos = block_reserve(vis.n, ws.q.count);
    for (uint32_t k = 0; k < vis.n; k++) {
      if (pos + k >= ws.q.capacity) {
        ct_latch_error(CT_ERR_CAPACITY, 9, screen_pos);
        break;
      }
      ws.q.a[pos + k] = vis.a[k];
      ws.q.b[pos + k] = vis.b[k];
      ws.q.c[pos + k] = vis.c[k];
    }
  }
  count_rays(P, rs);
}

// pass 2, ReSTIR PT block (rgen.glsl:427-452) and the rest of the shading
// (:453-509): spatial path reuse with pairwise RMIS
// (indirect_illumination.glsl:309-452)
// 4 blocks of 128 per SM (128 registers): 0.29 ms per 1080p frame against
// 0.33 ms with the register count left free (168) and 0.40 ms at 2 blocks
#ifndef CT_PT_SPATIAL_MIN_BLOCKS
#define CT_PT_SPATIAL_MIN_BLOCKS 4
#endif
template <bool HYBRID>
__global__ void __launch_bounds__(128, CT_PT_SPATIAL_MIN_BLOCKS) k_pt_spatial(ct_push_constant pc, DevAccel A, ct_params P) {
  __shared__ BlockConsts B;
  if (threadIdx.x == 0 && threadIdx.y == 0) load_frame_view(pc, B);
  __syncthreads();
  const FrameView &F = B.F;
  uint32_t x, y;
  pixel_of(x, y);
  RayStats rs = {};
  if (x < F.W && y < F.H) {
    const uint32_t screen_pos = y * F.W + x;
    const ct_di_info &dref = F.di[screen_pos];
    if (dref.distance > 0.0f) {
      rs.hits = 1;
      const PtParams pp = pt_params(F, P, A);
      const Isect cen_i = primary_isect(F, dref, true);
      const f3 camera_pos = f3{B.inv_view.c[3].x, B.inv_view.c[3].y, B.inv_view.c[3].z};
      ct_di_info &pref = F.prev_di[screen_pos];
      uint32_t seed = pref.seed;
      VisInline vis{A, screen_pos, rs};
      PathRes central = load_path_res(F.out_path_reservoir[screen_pos]);
      PathRes dst = path_res_init(pp.max_depth);
      const int32_t neighbor_count = (int32_t)pp.neighbor_count;
      int32_t valid_neighbor_count = 0;
      float canonical_weight = 1.f;
      const float cd = length(camera_pos - cen_i.world_hit);
      for (int32_t i = 0; i < neighbor_count; ++i) {
        // get_next_neighbor_pixel (prng.glsl:272-293)
        const float r1 = rnd(seed);
        const float r2 = rnd(seed);
        const float ox = 2.0f * r1 - 1.0f, oy = 2.0f * r2 - 1.0f;
        int32_t nx = (int32_t)x + f2i(ox * (float)pp.neighbor_radius);
        int32_t ny = (int32_t)y + f2i(oy * (float)pp.neighbor_radius);
        if (nx == (int32_t)x && ny == (int32_t)y) nx = ny = -1;
        if (!(nx < (int32_t)F.W && ny < (int32_t)F.H && nx >= 0 && ny >= 0)) continue;
        const uint32_t nidx = (uint32_t)ny * F.W + (uint32_t)nx;
        const ct_di_info &nd = F.di[nidx];
        if (!objhit_exists(nd.instance_hit.instance_id, nd.instance_hit.primitive_id)) continue;
        const Isect nb_i = primary_isect(F, nd, false);
        // is_valid_geometry (primitives.glsl:547-556)
        const float ndist = length(camera_pos - nb_i.world_hit);
        if (!(dot(cen_i.world_nrm, nb_i.world_nrm) >= 0.5f && fabsf(cd - ndist) < 0.1f * cd)) continue;
        const PathRes nres = load_path_res(F.out_path_reservoir[nidx]);
        rs.neighbours++;
        valid_neighbor_count++;
        float prefix_jacobian = 0.f;
        f3 prefix_integrand;
        if constexpr (HYBRID) {
          PathRes shifted = central;  // the shift may replace its cached Jacobian
          prefix_integrand =
              shift_hybrid(F, A, pp, prefix_jacobian, nb_i, cen_i, shifted, true, vis, 0u, InlineReplay{F, A, pp, screen_pos, rs});
        } else {
          prefix_integrand = shift_reconnection(F, A, prefix_jacobian, nb_i, cen_i, central, true, vis, 0u);
        }
        const float prefix_approx_pdf = path_scalar(prefix_integrand) * prefix_jacobian;
        canonical_weight += 1.f;
        if (prefix_approx_pdf > 0.f)
          canonical_weight -= prefix_approx_pdf * nres.M /
                              (prefix_approx_pdf * nres.M + central.M * path_scalar(central.F) / (float)neighbor_count);
        PathRes tdst = dst;
        float dst_jacobian = 0.f;
        const bool possible =
            shift_and_merge<HYBRID>(F, A, pp, dst_jacobian, cen_i, tdst, nb_i, nres, seed, vis, 1u,
                                    InlineReplay{F, A, pp, screen_pos, rs});
        float neighbor_weight = 0.f;
        if (possible) {
          neighbor_weight = path_scalar(nres.F) / dst_jacobian * nres.M /
                            ((path_scalar(nres.F) / dst_jacobian) * nres.M +
                             path_scalar(tdst.F) * central.M / (float)neighbor_count);
          if (isnan(neighbor_weight) || isinf(neighbor_weight)) neighbor_weight = 0.f;
        }
        path_res_merge_mis(dst, tdst.F, dst_jacobian, tdst, seed, neighbor_weight);
      }
      path_res_merge_mis(dst, central.F, 1.f, central, seed, canonical_weight);
      if (dst.weight > 0.f) {
        path_res_finalize_gris(dst);
        dst.weight = dst.weight / (float)(valid_neighbor_count + 1);
      }
      if (dst.weight < 0.f) dst.weight = 0.f;
      if (isnan(dst.weight) || isinf(dst.weight)) dst.weight = 0.f;
      const f3 indirect = dst.F * dst.weight;
      store_path_res(F.temporal_path_reservoir[screen_pos], dst);
      // hit_value = direct (left in the image by ct_restir_di) + indirect +
      // emission, non-finite channels to 0
      const float4 direct = F.swapchain[screen_pos];
      f3 hv = f3{direct.x, direct.y, direct.z};
      hv = hv + indirect;
      hv = hv + cen_i.mat.emission;
      if (isinf(hv.x) || isnan(hv.x)) hv.x = 0.0f;
      if (isinf(hv.y) || isnan(hv.y)) hv.y = 0.0f;
      if (isinf(hv.z) || isnan(hv.z)) hv.z = 0.0f;
      const float4 px = make_float4(hv.x, hv.y, hv.z, 1.0f);
      F.swapchain[screen_pos] = px;
      if (F.is_active & CT_TAA_BIT) F.taa_frame[screen_pos] = px;
      pref.seed = seed;
    }
  }
  count_rays(P, rs);
}

// ---------------------------------------------------------------------------
// batch queries (ct_trace_visibility / ct_trace_closest)
__global__ void __launch_bounds__(256) k_query_visibility(DevAccel A, const ct_ray_query *q, uint32_t n, uint8_t *out) {
  RayStats rs = {};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const ct_ray_query r = q[i];
    out[i] = vertex_visible(A, ld3(r.origin), ld3(r.direction), r.distance, r.target_instance, r.target_primitive,
                            (r.flags & CT_QUERY_CHECK_TARGET) != 0, i, rs) ? 1 : 0;
  }
}
__global__ void __launch_bounds__(256) k_query_closest(DevAccel A, const ct_ray_query *q, uint32_t n, ct_ray_hit *out) {
  RayStats rs = {};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const ct_ray_query r = q[i];
    HitRecord h = trace_primary(A, ld3(r.origin), ld3(r.direction), 0.0f, r.distance, i, rs);
    ct_ray_hit o;
    o.instance_id = h.hit ? h.inst : CT_MAX_INSTANCES;
    o.primitive_id = h.hit ? h.prim : CT_MAX_PRIMITIVES;
    o.t = h.hit ? h.t : -1.0f;
    o._pad = 0;
    out[i] = o;
  }
}
cudaError_t ct_launch_queries(const DevAccel &A, const ct_ray_query *q, uint32_t n, void *out, int closest,
                              cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const uint32_t blocks = (n + 255) / 256 < 65535 ? (n + 255) / 256 : 65535;
  if (closest) CT_TIMED(CT_K_QUERIES, s, k_query_closest<<<blocks, 256, 0, s>>>(A, q, n, (ct_ray_hit *)out));
  else CT_TIMED(CT_K_QUERIES, s, k_query_visibility<<<blocks, 256, 0, s>>>(A, q, n, (uint8_t *)out));
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launchers
static dim3 frame_grid(uint32_t W, uint32_t H, dim3 blk) {
  return dim3((W + blk.x - 1) / blk.x, (H + blk.y - 1) / blk.y, 1);
}

cudaError_t ct_launch_trace(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, cudaStream_t s) {
  dim3 blk(16, 8);
  CT_TIMED(CT_K_TRACE_PRIMARY, s, k_trace_primary<<<frame_grid(pc.size[0], pc.size[1], blk), blk, 0, s>>>(pc, A, P));
  return cudaGetLastError();
}
static Workspace make_ws(const CtWorkspace &w) {
  Workspace ws;
  ws.q.a = (float4 *)w.ray_a;
  ws.q.b = (float4 *)w.ray_b;
  ws.q.c = (uint2 *)w.ray_c;
  ws.q.count = w.counter;
  ws.q.capacity = w.capacity;
  ws.vis = w.vis;
  ws.rad = w.rad;
  ws.nbr = w.nbr;
  ws.smeta = (uint2 *)w.smeta;
  return ws;
}

static int sm_count() {
  static int n_sm = 0;
  if (n_sm == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    n_sm = v > 0 ? v : 148;
  }
  return n_sm;
}

// blocks of the persistent walkers: ct_params.walker_blocks, else 8 per SM
static uint32_t walker_grid(const ct_params &P) {
  return P.walker_blocks ? P.walker_blocks : (uint32_t)sm_count() * 8u;
}

// the frame accumulates work counters (CT_PARAM_COUNT_RAYS)
static bool counting(const ct_params &P) { return (P.flags & CT_PARAM_COUNT_RAYS) && P.counters_address; }

static cudaError_t trace_queue(const ct_push_constant &pc, const DevAccel &A, const ct_params &P,
                               const CtWorkspace &w, cudaStream_t s) {
  // the queue length is only known on the device: a grid that fills the GPU
  // walks the queue with a grid stride
  if (counting(P))
    CT_TIMED(CT_K_TRACE_SHADOW, s, k_trace_shadow<true><<<walker_grid(P), 256, 0, s>>>(A, P, make_ws(w)));
  else
    CT_TIMED(CT_K_TRACE_SHADOW, s, k_trace_shadow<false><<<walker_grid(P), 256, 0, s>>>(A, P, make_ws(w)));
  return cudaGetLastError();
}

cudaError_t ct_launch_di_stage0(const ct_push_constant &pc, const DevAccel &A, const DevAccel &A_prev,
                                const ct_params &P, const CtWorkspace &w, cudaStream_t s) {
  dim3 blk(16, 8);
  const dim3 grid = frame_grid(pc.size[0], pc.size[1], blk);
  const Workspace ws = make_ws(w);
  cudaError_t e;
  if ((e = cudaMemsetAsync(w.counter, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  CT_TIMED(CT_K_DI_GEN0, s, k_di_gen0<false><<<grid, blk, 0, s>>>(pc, P, ws, A));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  CT_TIMED(CT_K_DI_GEN0, s, k_di_gen0<true><<<grid, blk, 0, s>>>(pc, P, ws, A));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = trace_queue(pc, A, P, w, s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(w.counter, 0, (CT_PREV_COUNT + 1) * sizeof(uint32_t), s)) != cudaSuccess) return e;
  CT_TIMED(CT_K_DI_GEN1, s, k_di_gen1<<<grid, blk, 0, s>>>(pc, P, ws));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = trace_queue(pc, A, P, w, s)) != cudaSuccess) return e;
  CT_TIMED(CT_K_TRACE_PREV, s, k_trace_prev<<<sm_count() * 8, 128, 0, s>>>(pc, A_prev, P, ws));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  CT_TIMED(CT_K_DI_RESOLVE0, s, k_di_resolve0<<<grid, blk, 0, s>>>(pc, P, ws));
  return cudaGetLastError();
}

cudaError_t ct_launch_spatial_round(const ct_push_constant &pc, const DevAccel &A, const ct_params &P,
                                    const CtWorkspace &w, int src_sel, int final_pass, int dst_sel, cudaStream_t s) {
  dim3 blk(16, 8);
  const dim3 grid = frame_grid(pc.size[0], pc.size[1], blk);
  const Workspace ws = make_ws(w);
  cudaError_t e;
  if ((e = cudaMemsetAsync(w.counter, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  CT_TIMED(CT_K_SPATIAL_SELECT, s, k_spatial_select<<<grid, blk, 0, s>>>(pc, P, ws, src_sel));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  uint32_t nmax = P.max_num_of_neighbors > P.min_num_of_neighbors ? P.max_num_of_neighbors : P.min_num_of_neighbors;
  if (nmax > CT_MAX_NEIGHBORS) nmax = CT_MAX_NEIGHBORS;
  if (nmax > 0) {
    const uint32_t R = 2u * nmax;
    const uint64_t threads = (uint64_t)pc.size[0] * pc.size[1] * R;
    CT_TIMED(CT_K_SPATIAL_SAMPLE, s,
             k_spatial_sample<<<(uint32_t)((threads + CT_SPATIAL_SAMPLE_THREADS - 1) / CT_SPATIAL_SAMPLE_THREADS),
                                CT_SPATIAL_SAMPLE_THREADS, 0, s>>>(pc, P, ws, src_sel, R));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if ((e = trace_queue(pc, A, P, w, s)) != cudaSuccess) return e;
  CT_TIMED(CT_K_SPATIAL_RESOLVE, s, k_spatial_resolve<<<grid, blk, 0, s>>>(pc, P, ws, src_sel, final_pass, dst_sel));
  return cudaGetLastError();
}
cudaError_t ct_launch_taa(const ct_push_constant &pc, const ct_params &P, cudaStream_t s) {
  const uint32_t gx = pc.size[0] / 8, gy = pc.size[1] / 8;
  if (gx == 0 || gy == 0) return cudaSuccess;
  dim3 blk(8, 8);
  CT_TIMED(CT_K_TAA, s, k_taa<<<dim3(gx, gy, 1), blk, 0, s>>>(pc, P));
  return cudaGetLastError();
}

cudaError_t ct_launch_pt(const ct_push_constant &pc, const DevAccel &A, const ct_params &P, const CtWorkspace &w,
                         int stage, cudaStream_t s) {
  dim3 blk(16, 8);
  const dim3 grid = frame_grid(pc.size[0], pc.size[1], blk);
  if (stage != 0) {
    if (P.pt_shift_mapping == CT_SHIFT_HYBRID)
      CT_TIMED(CT_K_PT_SPATIAL, s, k_pt_spatial<true><<<grid, blk, 0, s>>>(pc, A, P));
    else
      CT_TIMED(CT_K_PT_SPATIAL, s, k_pt_spatial<false><<<grid, blk, 0, s>>>(pc, A, P));
    return cudaGetLastError();
  }
  PtWork pw;
  pw.state.col = (uint4 *)w.pt_state;
  pw.state.n = pc.size[0] * pc.size[1];
  pw.hit = (uint4 *)w.pt_hit;
  pw.q[0] = (float4 *)w.pt_q[0];
  pw.q[1] = (float4 *)w.pt_q[1];
  pw.count = w.counter + 8;
  pw.capacity = w.pt_capacity;
  pw.replay = (ReplayOut *)w.pt_replay;
  pw.jobs = (uint32_t *)w.pt_jobs;
  const Workspace ws = make_ws(w);
  cudaError_t e;
  if ((e = cudaMemsetAsync(pw.count, 0, 4 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  CT_TIMED(CT_K_PT_START, s, k_pt_start<<<grid, blk, 0, s>>>(pc, A, P, pw));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // the queue lengths are only known on the device: a fixed number of rounds,
  // enough for the longest path (max_depth < CT_PT_MAX_ITER), each a no-op
  // once the queues are empty.  A round queues at most one light-sample ray
  // per pixel and nothing reads their answers (a path's light sample only
  // counts towards PATH_RESERVOIR.M, which the path builder resets), so the
  // rays of `group` rounds share the shadow-ray queue and one walker launch.
  const uint64_t px = (uint64_t)pc.size[0] * pc.size[1];
  const int group = px && w.capacity / px > 0 ? (int)(w.capacity / px) : 1;
  if ((e = cudaMemsetAsync(w.counter, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  const int rounds = CT_PT_TAIL_ROUND < CT_PT_MAX_ITER ? CT_PT_TAIL_ROUND : CT_PT_MAX_ITER;
  for (int it = 0; it < rounds; it++) {
    const int qi = it & 1;
    if (counting(P))
      CT_TIMED(CT_K_PT_EXTEND, s, k_pt_extend<true><<<walker_grid(P), 256, 0, s>>>(A, P, pw, qi));
    else
      CT_TIMED(CT_K_PT_EXTEND, s, k_pt_extend<false><<<walker_grid(P), 256, 0, s>>>(A, P, pw, qi));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(pw.count + 2 * (qi ^ 1), 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
    CT_TIMED(CT_K_PT_SHADE, s, k_pt_shade<<<(walker_grid(P) + 1) / 2, 256, 0, s>>>(pc, A, P, ws, pw, qi));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((it + 1) % group == 0 || it + 1 == rounds) {
      if ((e = trace_queue(pc, A, P, w, s)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(w.counter, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
    }
  }
  if (rounds < CT_PT_MAX_ITER) {
    CT_TIMED(CT_K_PT_FINISH, s, k_pt_finish<<<walker_grid(P), 128, 0, s>>>(pc, A, P, ws, pw, rounds & 1));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = trace_queue(pc, A, P, w, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.counter, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
  }
  const bool hybrid = P.pt_shift_mapping == CT_SHIFT_HYBRID;
  if (hybrid) {
    // the replays temporal reuse will ask for, walked side by side first
    if ((e = cudaMemsetAsync(pw.count + 4, 0, sizeof(uint32_t), s)) != cudaSuccess) return e;
    CT_TIMED(CT_K_PT_REPLAY, s, k_pt_replay_jobs<<<grid, blk, 0, s>>>(pc, pw));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    CT_TIMED(CT_K_PT_REPLAY, s, k_pt_replay<<<sm_count() * 8, 128, 0, s>>>(pc, A, P, pw));
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (hybrid)
    CT_TIMED(CT_K_PT_TEMPORAL, s, k_pt_temporal<0, true><<<grid, blk, 0, s>>>(pc, A, P, ws, pw));
  else
    CT_TIMED(CT_K_PT_TEMPORAL, s, k_pt_temporal<0, false><<<grid, blk, 0, s>>>(pc, A, P, ws, pw));
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = trace_queue(pc, A, P, w, s)) != cudaSuccess) return e;
  if (hybrid)
    CT_TIMED(CT_K_PT_TEMPORAL, s, k_pt_temporal<1, true><<<grid, blk, 0, s>>>(pc, A, P, ws, pw));
  else
    CT_TIMED(CT_K_PT_TEMPORAL, s, k_pt_temporal<1, false><<<grid, blk, 0, s>>>(pc, A, P, ws, pw));
  return cudaGetLastError();
}

// device status word access for ct_get_error
cudaError_t ct_error_word_read(uint32_t *w, int reset, cudaStream_t s) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(w, g_ct_error, 4 * sizeof(uint32_t), 0, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess || !reset) return e;
  static const uint32_t z[4] = {0, 0, 0, 0};
  e = cudaMemcpyToSymbolAsync(g_ct_error, z, sizeof(z), 0, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

// scene edits (ct_brush / ct_rearrange)
#include "ct_edit.cuh"
#include "ct_adjoint.cuh"
