// oracle_main.cpp -- CPU parity oracle for the cube-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load the library built from this file; the
// product path (libct) never does.
//
// What runs here is the reference's own shader code: the GLSL of
// src/shaders/glsl/raytracing/rgen.glsl (both passes), rint.glsl, rchit.glsl
// (RIS_SELECTION), rmiss.glsl, rcall_scatter.glsl and compute/taa.glsl with
// everything they include, rewritten mechanically by oracle/transform.py and
// compiled against oracle/shim/glsl_shim.hpp.  This file adds what a Vulkan
// device would provide around that code:
//
//  * the ray-tracing pipeline: traceRayEXT runs the intersection shader on
//    every candidate voxel, keeps the closest reported hit and then runs the
//    closest-hit or miss shader (rgen.glsl:147-158, rint.glsl:10-43,
//    rchit.glsl:18-54, rmiss.glsl:25-28);
//  * ray queries (light.glsl:106-137, bounce.glsl:85-119): candidates are
//    presented in ascending order of the box-test distance the calling loop
//    computes, ties broken by the lowest primitive index.  With that order
//    the reference loops implement the hit rules the product kernels use:
//      - closest hit, ties -> lowest primitive index (traceRayEXT and
//        intersect());
//      - a shadow ray is blocked iff its first hit in that order inside
//        [0, distance] exists and is not the light's own voxel;
//  * candidate generation: a voxel-grid DDA in each instance's object space
//    that also offers the 26 neighbours of every visited cell, so rounding
//    in the box test can never hide a candidate from the rules above;
//  * the callable shaders table (main.cpp:730-757: 2 lambertian, 3 metal,
//    4 dielectric, 5 constant medium);
//  * the frame's dispatch shapes (main.cpp:1585-1645), including the TAA
//    dispatch of (W/8, H/8) groups of 8x8 that skips right/bottom edge
//    pixels when W or H is not a multiple of 8.
//
// Built twice (oracle/Makefile): in single precision, the parity oracle, and
// with CT_ORACLE_FP64 in double precision (ct_real), which states the error
// of the single-precision results.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <unordered_set>
#include <vector>
#include <thread>
#include <mutex>

#include "glsl_shim.hpp"

thread_local uvec3 gl_LaunchIDEXT;
thread_local uvec3 gl_LaunchSizeEXT;
thread_local uvec3 gl_GlobalInvocationID;
thread_local uvec3 gl_NumWorkGroups;
thread_local vec3 gl_WorldRayOriginEXT;
thread_local vec3 gl_WorldRayDirectionEXT;
thread_local mat4x3 gl_ObjectToWorldEXT;
thread_local int32_t gl_InstanceCustomIndexEXT;
thread_local int32_t gl_PrimitiveID;
thread_local ct_real gl_HitTEXT;

// capacity of SPATIAL_REUSE's neighbour list (transform.py rule 10); the
// CUDA path's CT_MAX_NEIGHBORS
#define CT_ORACLE_MAX_NEIGHBORS 8
#include "defines.glsl"

// Objects the GLSL declares with layout(...) qualifiers (push constant and
// ray payloads, defines.glsl:110-123).  One copy per host thread.
thread_local PushConstant p;
thread_local HIT_PAY_LOAD prd;
thread_local bool is_shadowed;
thread_local HIT_SCATTER_PAY_LOAD call_scatter;
thread_local HIT_MAT_PAY_LOAD hit_call;

#include "prng.glsl"
#include "primitives.glsl"
#include "mat.glsl"
#include "light.glsl"
#include "reservoir.glsl"
#include "indirect_illumination.glsl"
#include "restir_resampling.glsl"

// The shift mapping rgen.glsl passes in its scene parameters
// (transform.py rule 11): SHIFT_MAPPING_RECONNECTION, as the reference sets
// it, unless oracle_set_params selects the hybrid shift.
static daxa_u32 ct_pt_shift_mapping = SHIFT_MAPPING_RECONNECTION;

namespace rgen_pass1 {
#define RESTIR_PREPASS_AND_FIRST_VISIBILITY_TEST 1
#include "rgen.glsl"
#undef RESTIR_PREPASS_AND_FIRST_VISIBILITY_TEST
}  // namespace rgen_pass1

namespace rgen_pass2 {
#define THIRD_VISIBILITY_TEST_AND_SHADING_PASS 1
#include "rgen.glsl"
#undef THIRD_VISIBILITY_TEST_AND_SHADING_PASS
}  // namespace rgen_pass2

// The same two passes with the indirect-illumination (ReSTIR PT) blocks of
// rgen.glsl compiled in (defines.glsl:20 ships INDIRECT_ILLUMINATION_ON 0).
// Pass 1 of rgen.glsl uses `light_count` in its PT block without declaring it
// (rgen.glsl:281); pass 2 declares it as light_config.point_light_count
// (rgen.glsl:366).  The oracle supplies the same value to pass 1 through a
// namespace-scope variable, set per frame before the pass runs.
#undef INDIRECT_ILLUMINATION_ON
#define INDIRECT_ILLUMINATION_ON 1
namespace rgen_pt_pass1 {
daxa_u32 light_count;
#define RESTIR_PREPASS_AND_FIRST_VISIBILITY_TEST 1
#include "rgen.glsl"
#undef RESTIR_PREPASS_AND_FIRST_VISIBILITY_TEST
}  // namespace rgen_pt_pass1

namespace rgen_pt_pass2 {
#define THIRD_VISIBILITY_TEST_AND_SHADING_PASS 1
#include "rgen.glsl"
#undef THIRD_VISIBILITY_TEST_AND_SHADING_PASS
}  // namespace rgen_pt_pass2
#undef INDIRECT_ILLUMINATION_ON
#define INDIRECT_ILLUMINATION_ON 0

namespace rint_shader {
#include "rint.glsl"
}
namespace rchit_ris {
#define RIS_SELECTION 1
#include "rchit.glsl"
#undef RIS_SELECTION
}
namespace rmiss_shader {
#include "rmiss.glsl"
}
namespace rcall_lambertian {
#include "rcall_scatter.glsl"
}
namespace rcall_metal {
#define METAL 1
#include "rcall_scatter.glsl"
#undef METAL
}
namespace rcall_dielectric {
#define DIELECTRIC 1
#include "rcall_scatter.glsl"
#undef DIELECTRIC
}
namespace rcall_medium {
#define CONSTANT_MEDIUM 1
#include "rcall_scatter.glsl"
#undef CONSTANT_MEDIUM
}
// TAA's ALPHA (taa.glsl:13, 0.8 in the reference) as a run-time parameter
// (transform.py rule 10)
static daxa_f32 ct_taa_alpha = 0.8f;
namespace taa_shader {
#include "taa.glsl"
}

// ---------------------------------------------------------------------------
// The hybrid shift (oracle restatement; transform.py rule 11).  The
// reference switches it off (path_state.glsl:237, rgen.glsl:282, 437) and
// its version cannot run: the replay data it reads is stubbed
// (path_reservoir.glsl:37-58), its producer is commented out
// (indirect_illumination.glsl:300-302), a reconnection vertex at length 1
// is given an invalid predecessor (shift.glsl:377) and the result's
// Jacobian stays 0 (shift.glsl:362, 437).  With the hybrid shift selected, the base paths
// choose their reconnection vertex with the reference's own code (its
// hybrid branches of path_check_rc_vertex and the escaped-vertex marking);
// the shift itself is restated here, as the method defines it, and the
// CUDA path implements the same restatement (ct_pt.cuh, shift_hybrid):
//  * a path whose reconnection vertex is vertex 1 reconnects from the
//    destination's primary hit;
//  * a longer prefix is replayed from the destination's primary hit with
//    the source path's random numbers (its init_random_seed; one draw
//    skipped at every vertex where the base path sampled a light) up to the
//    vertex before the reconnection vertex, and reconnects from there with
//    the source side's pdfs and geometry term from its cached Jacobian;
//    the replay fails (not invertible) where a replayed vertex before that
//    one would itself qualify as reconnection vertex (far-field incoming
//    segment, rough, rough predecessor), where that vertex is not rough, or
//    where the replay misses or meets a zero throughput;
//  * the integrand is the replayed prefix throughput times the
//    reconnection's, the Jacobian the reconnection's (a replay is the
//    identity on random numbers);
//  * a path without a reconnection vertex does not shift.
// The replay is computed where the shift is evaluated, so `rc_data` is not
// read.
static bool ct_replay_prefix(const SCENE_PARAMS params, const INTERSECT dst, const PATH_RESERVOIR src,
                             daxa_u32 rc_length, INTERSECT &prev, daxa_f32vec3 &tp) {
  daxa_u32 seed = src.init_random_seed;
  INTERSECT i = dst;
  daxa_f32vec3 origin = compute_ray_origin(i.world_hit, i.world_nrm);
  origin = compute_ray_origin(origin, i.world_nrm);
  if (!generate_scatter_ray(i, seed)) return false;
  daxa_f32vec3 weight = evaluate_material(i.mat, i.world_nrm, i.wo, i.wi);
  daxa_f32 pdf = sample_material_pdf(i.mat, i.world_nrm, i.wo, i.wi);
  weight = weight / pdf;
  if (pdf <= 0.0f) return false;
  daxa_f32vec3 thp = weight;
  if (!(thp.x > 0.0f || thp.y > 0.0f || thp.z > 0.0f)) return false;
  daxa_f32vec3 dir = i.wi;
  daxa_b32 last_rough = true;  // the base path's value at its first bounce
  for (daxa_u32 len = 1; len < rc_length; len++) {
    INTERSECT h = intersect(Ray{origin, dir});
    if (!h.is_hit) return false;
    daxa_f32vec3 new_origin = compute_ray_origin(h.world_hit, h.world_nrm);
    new_origin = compute_ray_origin(new_origin, h.world_nrm);
    const daxa_b32 is_far_field = length(new_origin - origin) >= params.near_field_distance;
    const daxa_b32 rough = classify_as_rough(h.mat.roughness, params.roughness_threshold);
    if (is_far_field && rough && last_rough) return false;
    if (len + 1 == rc_length) {
      if (!rough) return false;
      prev = h;
      tp = thp;
      return true;
    }
    rnd(seed);
    if (!generate_scatter_ray(h, seed)) return false;
    weight = evaluate_material(h.mat, h.world_nrm, h.wo, h.wi);
    pdf = sample_material_pdf(h.mat, h.world_nrm, h.wo, h.wi);
    weight = weight / pdf;
    if (pdf <= 0.0f) return false;
    thp = thp * weight;
    if (!(thp.x > 0.0f || thp.y > 0.0f || thp.z > 0.0f)) return false;
    origin = new_origin;
    dir = h.wi;
    last_rough = rough;
  }
  return false;
}

daxa_f32vec3 compute_shifted_integrand_hybrid(const SCENE_PARAMS params, daxa_b32 use_prev,
                                              daxa_b32 temporal_update_for_dynamic_scene, daxa_f32 &dst_jacobian,
                                              const OBJECT_HIT dst_primary_hit,
                                              const INTERSECT dst_primary_intersection,
                                              const INTERSECT src_primary_intersection,
                                              PATH_RESERVOIR &temp_path_reservoir, RECONNECTION_DATA rc_data,
                                              daxa_b32 eval_visibility) {
  dst_jacobian = 0.f;
  if (temp_path_reservoir.weight == 0.f) return daxa_f32vec3(0.0f);
  const daxa_u32 rc_length = path_reservoir_get_reconnection_length(temp_path_reservoir.path_flags);
  const daxa_u32 path_length = path_reservoir_get_path_length(temp_path_reservoir.path_flags);
  const daxa_b32 escaped = path_length + 1 == rc_length;
  if (!(rc_length <= path_length || escaped) || !instance_hit_exists(temp_path_reservoir.rc_vertex_hit.object))
    return daxa_f32vec3(0.0f);
  INTERSECT prev = dst_primary_intersection;
  daxa_f32vec3 tp = daxa_f32vec3(1.0f);
  if (rc_length > 1 && !ct_replay_prefix(params, dst_primary_intersection, temp_path_reservoir, rc_length, prev, tp))
    return daxa_f32vec3(0.0f);
  PATH_RESERVOIR src = temp_path_reservoir;
  daxa_f32 jacobian = 0.f;
  const daxa_f32vec3 rc_tp = compute_shifted_integrand_reconnection(params, jacobian, prev, src_primary_intersection,
                                                                    src, eval_visibility, true, rc_length > 1);
  dst_jacobian = jacobian;
  temp_path_reservoir.cached_jacobian = src.cached_jacobian;
  return tp * rc_tp;
}

// ---------------------------------------------------------------------------
// Extra DI spatial rounds, for ct_params.spatial_passes > 1.  The reference
// compiles one round into its shading pass; this extension of the oracle
// mirrors the CUDA path's rounds.  With n rounds, extra round r (r < n - 1)
// reads the reservoirs of one buffer and writes the other: intermediate ->
// current (RESTIR.reservoir_address) -> intermediate ...; the shading pass
// then runs with the last round's output bound as the intermediate buffer.
// Per hit pixel a round runs the shading pass's own set-up and its
// SPATIAL_REUSE call (rgen.glsl:330-397) with the source buffer bound as the
// intermediate reservoirs, stores the reservoir in the destination buffer
// and the seed SPATIAL_REUSE advanced in the pixel's DI record (after the
// round, so that no pixel reads a neighbour's record mid-round); it shades
// nothing and leaves missed pixels alone.
struct SpatialRoundOut {
  RESERVOIR *dst;
  std::vector<std::pair<uint32_t, uint32_t>> seeds;  // (pixel, seed)
};
static thread_local SpatialRoundOut *tl_round;

static void spatial_round_main() {
  const daxa_i32vec2 index = ivec2{gl_LaunchIDEXT.xy()};
  const daxa_u32vec2 rt_size = gl_LaunchSizeEXT.xy();
  const daxa_u32 screen_pos = index.y * rt_size.x + index.x;
  DIRECT_ILLUMINATION_INFO di_info = get_di_from_current_frame(screen_pos);
  if (!(di_info.distance > 0.0f)) return;
  Ray ray = Ray{di_info.ray_origin, normalize(di_info.position - di_info.ray_origin)};
  MATERIAL mat = get_material_from_material_index(di_info.mat_index);
  LIGHT_CONFIG light_config = get_light_config_from_light_index();
  daxa_u32 light_count = light_config.point_light_count;
  HIT_INFO_INPUT hit = HIT_INFO_INPUT{di_info.position, di_info.normal, di_info.distance, daxa_f32vec3{0.f},
                                      di_info.instance_hit, di_info.mat_index};
  hit.world_hit = compute_ray_origin(hit.world_hit, hit.world_nrm);
  hit.world_hit = compute_ray_origin(hit.world_hit, hit.world_nrm);
  daxa_f32 pdf = 1.0f / glsl_f32(light_count);
  RESERVOIR reservoir = get_reservoir_from_intermediate_frame_by_index(screen_pos);
  SPATIAL_REUSE(reservoir, di_info.confidence, index, rt_size, ray, hit, di_info.mat_index, mat, light_count, pdf,
                di_info.seed, MIN_NEIGHBORS_RADIUS, MAX_NEIGHBORS_RADIUS);
  tl_round->dst[screen_pos] = reservoir;
  tl_round->seeds.emplace_back(screen_pos, di_info.seed);
}

// ---------------------------------------------------------------------------
// scene: one dense voxel grid per instance, voxel -> lowest primitive id
struct OracleGrid {
  int ox, oy, oz;       // voxel coordinate of cell (0,0,0)
  int nx, ny, nz;
  std::vector<int32_t> prim;  // -1 = empty
  int32_t at(int x, int y, int z) const {
    x -= ox; y -= oy; z -= oz;
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return -1;
    return prim[((size_t)z * ny + y) * nx + x];
  }
};
struct OracleAccel {
  std::vector<INSTANCE> instances;
  std::vector<OracleGrid> grids;
  std::vector<AABB> aabbs;  // the boxes it was built from
  float extent;
  bool previous = false;    // bound as p.tlas_previous after a scene edit
};

struct RayCounters {
  uint64_t primary = 0, shadow = 0, bounce = 0, box_tests = 0, bricks = 0;
};
static thread_local RayCounters tl_count;
static RayCounters g_count;

// Enumerate candidate voxels of one instance along a ray given in that
// instance's object space.  visit(prim) returns the candidate's hit distance
// (or +inf); enumeration stops two cells after the cells' entry distance has
// passed both the best distance returned so far and t_stop.
template <class Visit>
static void enumerate_candidates(const OracleGrid &g, double extent, vec3 o_obj, vec3 d_obj, double tmin,
                                 double t_stop, Visit visit) {
  double o[3] = {o_obj.x / extent, o_obj.y / extent, o_obj.z / extent};
  double d[3] = {d_obj.x / extent, d_obj.y / extent, d_obj.z / extent};
  double lo[3] = {(double)g.ox - 1, (double)g.oy - 1, (double)g.oz - 1};
  double hi[3] = {(double)(g.ox + g.nx + 1), (double)(g.oy + g.ny + 1), (double)(g.oz + g.nz + 1)};
  double t0 = tmin, t1 = t_stop;
  for (int a = 0; a < 3; a++) {
    if (d[a] == 0.0) {
      if (o[a] < lo[a] || o[a] > hi[a]) return;
    } else {
      double ta = (lo[a] - o[a]) / d[a], tb = (hi[a] - o[a]) / d[a];
      if (ta > tb) std::swap(ta, tb);
      t0 = std::max(t0, ta);
      t1 = std::min(t1, tb);
    }
  }
  if (t0 > t1 + 1e-9) return;
  int c[3], step[3];
  double tmax[3], tdelta[3];
  for (int a = 0; a < 3; a++) {
    double pos = o[a] + d[a] * t0;
    c[a] = (int)std::floor(pos);
    c[a] = std::min(std::max(c[a], (int)lo[a]), (int)hi[a] - 1);
    if (d[a] > 0) { step[a] = 1; tmax[a] = (c[a] + 1 - o[a]) / d[a]; tdelta[a] = 1.0 / d[a]; }
    else if (d[a] < 0) { step[a] = -1; tmax[a] = (c[a] - o[a]) / d[a]; tdelta[a] = -1.0 / d[a]; }
    else { step[a] = 0; tmax[a] = INFINITY; tdelta[a] = INFINITY; }
  }
  std::unordered_set<int64_t> seen;
  double best = INFINITY;
  double entry = t0;
  int extra = 0;
  int last_brick = INT32_MIN;
  for (int iter = 0; iter < 1 << 22; iter++) {
    if (entry > t_stop || entry > best) {
      if (++extra > 2) break;
    }
    int brick = ((c[2] >> 3) * 4099 + (c[1] >> 3)) * 4099 + (c[0] >> 3);
    if (brick != last_brick) { tl_count.bricks++; last_brick = brick; }
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
          int32_t pr = g.at(x, y, z);
          if (pr < 0) continue;
          int64_t key = ((int64_t)(z + 4096) << 40) | ((int64_t)(y + 4096) << 20) | (int64_t)(x + 4096);
          if (!seen.insert(key).second) continue;
          tl_count.box_tests++;
          double t = visit(pr);
          if (t < best) best = t;
        }
    int a = (tmax[0] < tmax[1]) ? (tmax[0] < tmax[2] ? 0 : 2) : (tmax[1] < tmax[2] ? 1 : 2);
    entry = tmax[a];
    c[a] += step[a];
    tmax[a] += tdelta[a];
    if (c[a] < (int)lo[a] || c[a] >= (int)hi[a]) break;
  }
}

static inline mat4x3 to_4x3(const mat4 &m) {
  mat4x3 r;
  for (int i = 0; i < 4; i++) r.c[i] = vec3(m.c[i].x, m.c[i].y, m.c[i].z);
  return r;
}

// rule: (t, global primitive index) lexicographic minimum
struct Best {
  bool hit = false;
  ct_real t = 0;
  uint32_t inst = 0, prim = 0, global = 0;
  bool better(ct_real tt, uint32_t g) const { return !hit || tt < t || (tt == t && g < global); }
};

static thread_local Best tl_report_best;
static thread_local ct_real tl_report_tmin, tl_report_tmax;
static thread_local uint32_t tl_report_inst, tl_report_prim, tl_report_global;

bool reportIntersectionEXT(ct_real t, uint32_t) {
  ct_real tmax = tl_report_best.hit ? tl_report_best.t : tl_report_tmax;
  if (!(t >= tl_report_tmin && t <= tmax)) return false;
  if (tl_report_best.better(t, tl_report_global)) {
    tl_report_best.hit = true;
    tl_report_best.t = t;
    tl_report_best.inst = tl_report_inst;
    tl_report_best.prim = tl_report_prim;
    tl_report_best.global = tl_report_global;
  }
  return true;
}

void traceRayEXT(daxa_TlasId tlas, uint32_t, uint32_t, uint32_t sbt_offset, uint32_t, uint32_t, vec3 origin, ct_real tmin,
                 vec3 dir, ct_real tmax, int) {
  tl_count.primary++;
  const OracleAccel &acc = *tlas;
  tl_report_best = Best();
  tl_report_tmin = tmin;
  tl_report_tmax = tmax;
  for (uint32_t ii = 0; ii < acc.instances.size(); ii++) {
    const INSTANCE &inst = acc.instances[ii];
    mat4 w2o = inverse(inst.transform);
    vec3 o_obj = (w2o * vec4(origin, 1.0f)).xyz();
    vec3 d_obj = (w2o * vec4(dir, 0.0f)).xyz();
    mat4x3 o2w = to_4x3(inst.transform);
    enumerate_candidates(acc.grids[ii], acc.extent, o_obj, d_obj, tmin, tmax, [&](int32_t pr) -> double {
      gl_WorldRayOriginEXT = origin;
      gl_WorldRayDirectionEXT = dir;
      gl_ObjectToWorldEXT = o2w;
      gl_InstanceCustomIndexEXT = (int32_t)ii;
      gl_PrimitiveID = pr;
      tl_report_inst = ii;
      tl_report_prim = (uint32_t)pr;
      tl_report_global = inst.first_primitive_index + (uint32_t)pr;
      rint_shader::main();
      return tl_report_best.hit ? (double)tl_report_best.t : INFINITY;
    });
  }
  gl_WorldRayOriginEXT = origin;
  gl_WorldRayDirectionEXT = dir;
  if (tl_report_best.hit) {
    const INSTANCE &inst = acc.instances[tl_report_best.inst];
    gl_ObjectToWorldEXT = to_4x3(inst.transform);
    gl_InstanceCustomIndexEXT = (int32_t)tl_report_best.inst;
    gl_PrimitiveID = (int32_t)tl_report_best.prim;
    gl_HitTEXT = tl_report_best.t;
    if (sbt_offset == 0) rchit_ris::main();
    else { fprintf(stderr, "oracle: hit group %u not available\n", sbt_offset); abort(); }
  } else {
    rmiss_shader::main();
  }
}

rayQueryEXT::~rayQueryEXT() { delete[] cand; delete[] cand_inst; }

void rayQueryInitializeEXT(rayQueryEXT &q, daxa_TlasId tlas, uint32_t flags, uint32_t, vec3 origin, ct_real tmin, vec3 dir,
                           ct_real tmax) {
  q.tlas = tlas; q.flags = flags; q.origin = origin; q.dir = dir; q.tmin = tmin; q.tmax = tmax;
  q.next = 0; q.committed = false; q.terminated = false;
  const bool visibility = (flags & gl_RayFlagsTerminateOnFirstHitEXT) != 0;
  if (visibility) tl_count.shadow++; else tl_count.bounce++;
  // The calling loops test candidates with is_hit_from_ray on
  //  - the query ray itself, rays may not start inside a box (light.glsl:121)
  //  - the query ray with its origin moved by compute_ray_origin(origin, dir),
  //    rays may start inside a box (bounce.glsl:211, 297).
  Ray key_ray = Ray{visibility ? origin : compute_ray_origin(origin, dir), dir};
  const bool can_start = !visibility;
  const OracleAccel &acc = *tlas;
  struct C { ct_real t; uint32_t g, inst, prim; };
  std::vector<C> hits;
  ct_real best = INFINITY;
  for (uint32_t ii = 0; ii < acc.instances.size(); ii++) {
    const INSTANCE &inst = acc.instances[ii];
    mat4 w2o = inverse(inst.transform);
    vec3 o_obj = (w2o * vec4(origin, 1.0f)).xyz();
    vec3 d_obj = (w2o * vec4(dir, 0.0f)).xyz();
    enumerate_candidates(acc.grids[ii], acc.extent, o_obj, d_obj, tmin, tmax, [&](int32_t pr) -> double {
      ct_real t;
      vec3 pos, nor;
      mat4 model, inv_model;
      if (acc.previous) {
        // A structure built before a scene edit reports the primitives whose
        // box at build time the ray hits (a BVH over the previous AABBs);
        // the shader then tests the current AABB of that id.  The walk
        // cannot stop at the nearest current hit: it runs to t_max.
        const AABB &b = acc.aabbs[inst.first_primitive_index + (uint32_t)pr];
        const vec3 h = daxa_f32vec3(HALF_VOXEL_EXTENT);
        Box box = Box((b.minimum + b.maximum) * 0.5f, h, safeInverse(h), mat3(1.f));
        Ray obj_ray = Ray{(w2o * vec4(key_ray.origin, 1.0f)).xyz(), d_obj};
        ct_real t_old;
        vec3 n_old;
        if (!intersect_box(box, obj_ray, t_old, n_old, can_start, false, safeInverse(obj_ray.direction)) ||
            !(t_old >= 0.0f && t_old <= tmax))
          return INFINITY;
        if (is_hit_from_ray(key_ray, OBJECT_INFO{ii, (uint32_t)pr}, daxa_f32vec3(HALF_VOXEL_EXTENT), t, pos, nor,
                            model, inv_model, false, can_start, true))
          hits.push_back(C{t, inst.first_primitive_index + (uint32_t)pr, ii, (uint32_t)pr});
        return INFINITY;
      }
      if (!is_hit_from_ray(key_ray, OBJECT_INFO{ii, (uint32_t)pr}, daxa_f32vec3(HALF_VOXEL_EXTENT), t, pos, nor, model,
                           inv_model, false, can_start, true))
        return best;
      hits.push_back(C{t, inst.first_primitive_index + (uint32_t)pr, ii, (uint32_t)pr});
      if (t < best) best = t;
      return best;
    });
  }
  std::sort(hits.begin(), hits.end(), [](const C &a, const C &b) { return a.t < b.t || (a.t == b.t && a.g < b.g); });
  delete[] q.cand; delete[] q.cand_inst;
  q.n = (uint32_t)hits.size();
  q.cand = new uint32_t[q.n > 0 ? q.n : 1];
  q.cand_inst = new uint32_t[q.n > 0 ? q.n : 1];
  for (uint32_t i = 0; i < q.n; i++) { q.cand[i] = hits[i].prim; q.cand_inst[i] = hits[i].inst; }
}

bool rayQueryProceedEXT(rayQueryEXT &q) {
  if (q.terminated) return false;
  if ((q.flags & gl_RayFlagsTerminateOnFirstHitEXT) && q.committed) return false;
  if (q.next >= q.n) return false;
  q.cur = q.next++;
  return true;
}
uint32_t rayQueryGetIntersectionTypeEXT(rayQueryEXT &q, bool committed) {
  if (committed) return q.committed ? gl_RayQueryCommittedIntersectionGeneratedEXT : gl_RayQueryCommittedIntersectionNoneEXT;
  return gl_RayQueryCandidateIntersectionAABBEXT;
}
int32_t rayQueryGetIntersectionInstanceCustomIndexEXT(rayQueryEXT &q, bool) { return (int32_t)q.cand_inst[q.cur]; }
int32_t rayQueryGetIntersectionPrimitiveIndexEXT(rayQueryEXT &q, bool) { return (int32_t)q.cand[q.cur]; }
void rayQueryGenerateIntersectionEXT(rayQueryEXT &q, ct_real t) {
  ct_real tmax = q.committed ? q.committed_t : q.tmax;
  if (t >= q.tmin && t <= tmax) { q.committed = true; q.committed_t = t; }
}
void rayQueryTerminateEXT(rayQueryEXT &q) { q.terminated = true; }

void executeCallableEXT(uint32_t sbt_index, uint32_t) {
  switch (sbt_index) {
    case 2: rcall_lambertian::main(); break;
    case 3: rcall_metal::main(); break;
    case 4: rcall_dielectric::main(); break;
    case 5: rcall_medium::main(); break;
    default: fprintf(stderr, "oracle: callable %u not available\n", sbt_index); abort();
  }
}

// ---------------------------------------------------------------------------
// C entry points (ctypes)
extern "C" {

struct OracleInfo {
  uint32_t sizeof_instance, sizeof_aabb, sizeof_primitive, sizeof_material, sizeof_light, sizeof_light_config,
      sizeof_reservoir, sizeof_di_info, sizeof_velocity, sizeof_path_reservoir, sizeof_camera_view, sizeof_status,
      sizeof_world, sizeof_restir, sizeof_push_constant;
  float voxel_extent;
};

void oracle_info(OracleInfo *info) {
  info->sizeof_instance = sizeof(INSTANCE);
  info->sizeof_aabb = sizeof(AABB);
  info->sizeof_primitive = sizeof(PRIMITIVE);
  info->sizeof_material = sizeof(MATERIAL);
  info->sizeof_light = sizeof(LIGHT);
  info->sizeof_light_config = sizeof(LIGHT_CONFIG);
  info->sizeof_reservoir = sizeof(RESERVOIR);
  info->sizeof_di_info = sizeof(DIRECT_ILLUMINATION_INFO);
  info->sizeof_velocity = sizeof(VELOCITY);
  info->sizeof_path_reservoir = sizeof(PATH_RESERVOIR);
  info->sizeof_camera_view = sizeof(camera_view);
  info->sizeof_status = sizeof(Status);
  info->sizeof_world = sizeof(WORLD);
  info->sizeof_restir = sizeof(RESTIR);
  info->sizeof_push_constant = sizeof(PushConstant);
  info->voxel_extent = VOXEL_EXTENT;
}

// Returns nullptr when an AABB is not one grid-aligned voxel.
void *oracle_build_accel(const INSTANCE *instances, uint32_t n_instances, const AABB *aabbs, uint32_t n_aabbs) {
  OracleAccel *acc = new OracleAccel();
  acc->extent = VOXEL_EXTENT;
  acc->aabbs.assign(aabbs, aabbs + n_aabbs);
  const double e = VOXEL_EXTENT;
  for (uint32_t ii = 0; ii < n_instances; ii++) {
    const INSTANCE &inst = instances[ii];
    acc->instances.push_back(inst);
    OracleGrid g;
    int mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    std::vector<int> coords(3 * (size_t)inst.primitive_count);
    for (uint32_t k = 0; k < inst.primitive_count; k++) {
      uint32_t gi = inst.first_primitive_index + k;
      if (gi >= n_aabbs) { delete acc; return nullptr; }
      const AABB &b = aabbs[gi];
      double lo[3] = {b.minimum.x, b.minimum.y, b.minimum.z}, up[3] = {b.maximum.x, b.maximum.y, b.maximum.z};
      for (int a = 0; a < 3; a++) {
        double v = lo[a] / e;
        int iv = (int)std::lround(v);
        if (std::fabs(v - iv) > 1e-4 || std::fabs((up[a] - lo[a]) / e - 1.0) > 1e-4) { delete acc; return nullptr; }
        coords[3 * k + a] = iv;
        mn[a] = std::min(mn[a], iv);
        mx[a] = std::max(mx[a], iv);
      }
    }
    if (inst.primitive_count == 0) { mn[0] = mn[1] = mn[2] = 0; mx[0] = mx[1] = mx[2] = 0; }
    g.ox = mn[0]; g.oy = mn[1]; g.oz = mn[2];
    g.nx = mx[0] - mn[0] + 1; g.ny = mx[1] - mn[1] + 1; g.nz = mx[2] - mn[2] + 1;
    g.prim.assign((size_t)g.nx * g.ny * g.nz, -1);
    for (uint32_t k = 0; k < inst.primitive_count; k++) {
      size_t idx = ((size_t)(coords[3 * k + 2] - g.oz) * g.ny + (coords[3 * k + 1] - g.oy)) * g.nx + (coords[3 * k] - g.ox);
      if (g.prim[idx] < 0) g.prim[idx] = (int32_t)k;  // lowest primitive id wins
    }
    acc->grids.push_back(std::move(g));
  }
  return acc;
}

void oracle_free_accel(void *acc) { delete (OracleAccel *)acc; }
void oracle_accel_set_previous(void *acc, int previous) { ((OracleAccel *)acc)->previous = previous != 0; }

// The run-time values of the reference constants transform.py rules 10 and
// 11 turn into variables, in ct_params' units.  `u` holds the counts
// (MIN/MAX_RIS_POINT/ENV/CUBE_SAMPLE_COUNT, MIN/MAX_NUM_OF_NEIGHBORS,
// NEIGHBOR_COUNT, NEIGHBOR_RADIUS, the shift mapping), `f` the reals
// (MIN/MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD, MIN/MAX_NEIGHBORS_RADIUS,
// MAX_DISTANCE_TO_HIT, MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD_PT, TAA ALPHA,
// NEAR_FIELD_DISTANCE with 0 for the reference's HALF_VOXEL_EXTENT * 0.5),
// as single-precision values, which the FP64 build widens.  Returns 1 when
// a neighbour count exceeds CT_ORACLE_MAX_NEIGHBORS or the shift mapping is
// neither reconnection nor hybrid, else 0.
int oracle_set_params(const uint32_t *u, const float *f) {
  if (u[6] > CT_ORACLE_MAX_NEIGHBORS || u[7] > CT_ORACLE_MAX_NEIGHBORS) return 1;
  if (u[10] != SHIFT_MAPPING_RECONNECTION && u[10] != SHIFT_MAPPING_HYBRID) return 1;
  ct_pt_shift_mapping = u[10];
  NEAR_FIELD_DISTANCE = f[7] > 0.0f ? (daxa_f32)f[7] : HALF_VOXEL_EXTENT * 0.5f;
  MIN_RIS_POINT_SAMPLE_COUNT = u[0];
  MAX_RIS_POINT_SAMPLE_COUNT = u[1];
  MIN_RIS_ENV_SAMPLE_COUNT = u[2];
  MAX_RIS_ENV_SAMPLE_COUNT = u[3];
  MIN_RIS_CUBE_SAMPLE_COUNT = u[4];
  MAX_RIS_CUBE_SAMPLE_COUNT = u[5];
  MIN_NUM_OF_NEIGHBORS = u[6];
  MAX_NUM_OF_NEIGHBORS = u[7];
  NEIGHBOR_COUNT = (daxa_i32)u[8];
  NEIGHBOR_RADIUS = (daxa_i32)u[9];
  MIN_INFLUENCE_FROM_THE_PAST_THRESHOLD = f[0];
  MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD = f[1];
  MIN_NEIGHBORS_RADIUS = f[2];
  MAX_NEIGHBORS_RADIUS = f[3];
  MAX_DISTANCE_TO_HIT = f[4];
  MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD_PT = f[5];
  ct_taa_alpha = f[6];
  return 0;
}

// which: 1 = ray-gen pass 1 (primary visibility, RIS, temporal reuse),
//        2 = ray-gen pass 2 (spatial reuse, shading),
//        3 = TAA compute pass,
//        4 / 5 = an extra DI spatial round (spatial_round_main) from the
//            intermediate to the current reservoirs / the other way,
//        11 / 12 = passes 1 / 2 with ReSTIR PT compiled in.
// Runs the pass over the rows [row_begin, row_end) (all rows when
// row_end == 0).  Returns 0.
int oracle_pass(int which, const PushConstant *pc, int nthreads, uint32_t row_begin, uint32_t row_end) {
  const uint32_t W = pc->size.x, H = pc->size.y;
  if (row_end == 0 || row_end > H) row_end = H;
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  uint32_t y_end = row_end;
  if (which == 3) y_end = std::min(row_end, (H / 8) * 8);
  if (which == 11) {
    const Status *status = (const Status *)(uintptr_t)pc->status_buffer;
    const LIGHT_CONFIG *lc = (const LIGHT_CONFIG *)(uintptr_t)status->light_config_address;
    rgen_pt_pass1::light_count = lc->point_light_count;
  }
  // an extra spatial round runs with its source bound as the intermediate
  // reservoir buffer
  PushConstant round_pc = *pc;
  RESTIR round_restir = *pc->restir_buffer;
  RESERVOIR *round_dst = nullptr;
  if (which == 4 || which == 5) {
    const daxa_u64 int_addr = round_restir.intermediate_reservoir_address, cur_addr = round_restir.reservoir_address;
    round_restir.intermediate_reservoir_address = which == 4 ? int_addr : cur_addr;
    round_dst = (RESERVOIR *)(uintptr_t)(which == 4 ? cur_addr : int_addr);
    round_pc.restir_buffer = &round_restir;
  }
  std::vector<std::pair<uint32_t, uint32_t>> round_seeds;
  std::atomic<uint32_t> next_row{row_begin};
  std::mutex mu;
  RayCounters total;
  auto worker = [&]() {
    p = round_pc;
    tl_count = RayCounters();
    SpatialRoundOut round_out{round_dst, {}};
    tl_round = &round_out;
    for (;;) {
      uint32_t y = next_row.fetch_add(1);
      if (y >= y_end) break;
      if (which == 4 || which == 5) {
        for (uint32_t x = 0; x < W; x++) {
          gl_LaunchIDEXT = uvec3(x, y, 0u);
          gl_LaunchSizeEXT = uvec3(W, H, 1u);
          spatial_round_main();
        }
      } else if (which == 1 || which == 2 || which == 11 || which == 12) {
        for (uint32_t x = 0; x < W; x++) {
          // ray payloads start out undefined on a device; here they start zeroed
          prd = HIT_PAY_LOAD{};
          call_scatter = HIT_SCATTER_PAY_LOAD{};
          gl_LaunchIDEXT = uvec3(x, y, 0u);
          gl_LaunchSizeEXT = uvec3(W, H, 1u);
          switch (which) {
            case 1: rgen_pass1::main(); break;
            case 2: rgen_pass2::main(); break;
            case 11: rgen_pt_pass1::main(); break;
            default: rgen_pt_pass2::main(); break;
          }
        }
      } else if (which == 3) {
        const uint32_t gx = W / 8, gy = H / 8;
        for (uint32_t x = 0; x < gx * 8; x++) {
          gl_GlobalInvocationID = uvec3(x, y, 0u);
          gl_NumWorkGroups = uvec3(gx, gy, 1u);
          taa_shader::main();
        }
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    total.primary += tl_count.primary; total.shadow += tl_count.shadow; total.bounce += tl_count.bounce;
    total.box_tests += tl_count.box_tests; total.bricks += tl_count.bricks;
    round_seeds.insert(round_seeds.end(), round_out.seeds.begin(), round_out.seeds.end());
    tl_round = nullptr;
  };
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  if (which == 4 || which == 5) {
    DIRECT_ILLUMINATION_INFO *di = (DIRECT_ILLUMINATION_INFO *)(uintptr_t)round_restir.di_address;
    for (const auto &ps : round_seeds) di[ps.first].seed = ps.second;
  }
  g_count.primary += total.primary; g_count.shadow += total.shadow; g_count.bounce += total.bounce;
  g_count.box_tests += total.box_tests; g_count.bricks += total.bricks;
  return 0;
}

// Ray counters accumulated over all passes since the last reset:
// out[0] primary, out[1] shadow (visibility queries), out[2] bounce queries,
// out[3] box tests, out[4] voxel-cell visits that changed 8^3 brick.
// ct_fpmath.h as the shim sees it (sin, cos, pow(x, 5)), for its error test
void oracle_fpmath(const float *x, uint32_t n, float *s, float *c, float *p5) {
  for (uint32_t i = 0; i < n; i++) { s[i] = sin(x[i]); c[i] = cos(x[i]); p5[i] = pow(x[i], 5.0f); }
}

void oracle_counters(uint64_t *out, int reset) {
  out[0] = g_count.primary; out[1] = g_count.shadow; out[2] = g_count.bounce;
  out[3] = g_count.box_tests; out[4] = g_count.bricks;
  if (reset) g_count = RayCounters();
}

// Ray queries with the reference's own functions: is_vertex_visible
// (light.glsl:82-142) and traceRayEXT with the intersection shader
// (rint.glsl), on records laid out as ct_ray_query (40 B: origin[3],
// distance, direction[3], flags, target instance, target primitive).
// out: uint8 visibility, or ct_ray_hit (instance, primitive, t, pad).
int oracle_queries(int closest, const PushConstant *pc, const void *records, uint32_t n, void *out, int nthreads) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<uint32_t> next{0};
  auto worker = [&]() {
    p = *pc;
    for (;;) {
      uint32_t i = next.fetch_add(64);
      if (i >= n) break;
      for (uint32_t k = i; k < std::min(n, i + 64); k++) {
        const float *r = (const float *)((const char *)records + 40ull * k);
        const uint32_t *u = (const uint32_t *)r;
        vec3 o(r[0], r[1], r[2]), d(r[4], r[5], r[6]);
        if (closest) {
          prd = HIT_PAY_LOAD{};
          traceRayEXT(p.tlas, 0u, 0xFFu, 0u, 0u, 0u, o, 0.0f, d, r[3], 0);
          uint32_t *h = (uint32_t *)((char *)out + 16ull * k);
          h[0] = tl_report_best.hit ? tl_report_best.inst : MAX_INSTANCES;
          h[1] = tl_report_best.hit ? tl_report_best.prim : MAX_PRIMITIVES;
          float t = tl_report_best.hit ? tl_report_best.t : -1.0f;
          memcpy(&h[2], &t, 4);
          h[3] = 0;
        } else {
          bool v = is_vertex_visible(Ray{o, d}, r[3], OBJECT_INFO{u[8], u[9]}, (u[7] & 1u) != 0, false);
          ((uint8_t *)out)[k] = v ? 1 : 0;
        }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  return 0;
}

// The paths of the adjoint renderer (ct_adjoint_forward / ct_adjoint_backward,
// include/ct.h; no reference counterpart), traced with the reference's own
// ray functions: the pinhole ray of get_ray_from_current_pixel
// (rgen.glsl:18-42) with the pixel centre moved by two draws of the sample's
// LCG (random.glsl:43-77, seeded with tea(pixel, seed + s)) instead of 0.5,
// closest hits of intersect() (bounce.glsl:9-125), the hit point moved off
// the surface twice (compute_ray_origin, primitives.glsl:233-257), and the
// Lambertian callable's direction (random_cosine_direction,
// rcall_scatter.glsl:74-86).  Writes, for every pixel of rect (x0, y0, x1,
// y1) row by row and every sample, `depth` global primitive indices
// (INSTANCE.first_primitive_index + primitive id) of the path's vertices,
// 0xFFFFFFFF after its end.  The radiance and gradients are computed from
// these paths by the caller, in the precision it wants.
int oracle_adjoint_paths(const PushConstant *pc, const float *inv_view16, const float *inv_proj16, uint32_t W,
                         uint32_t H, uint32_t spp, uint32_t depth, uint32_t seed, const uint32_t *rect,
                         uint32_t *verts, int nthreads) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  const uint32_t x0 = rect[0], y0 = rect[1], x1 = rect[2], y1 = rect[3];
  if (x0 >= x1 || y0 >= y1 || x1 > W || y1 > H || depth == 0) return 1;
  mat4 inv_view, inv_proj;
  for (int c = 0; c < 4; c++) {
    inv_view.c[c] = vec4(inv_view16[4 * c], inv_view16[4 * c + 1], inv_view16[4 * c + 2], inv_view16[4 * c + 3]);
    inv_proj.c[c] = vec4(inv_proj16[4 * c], inv_proj16[4 * c + 1], inv_proj16[4 * c + 2], inv_proj16[4 * c + 3]);
  }
  const uint32_t rw = x1 - x0;
  std::atomic<uint32_t> next{y0};
  auto worker = [&]() {
    p = *pc;
    const INSTANCE *instances = (const INSTANCE *)(uintptr_t)deref(p.world_buffer).instance_address;
    for (;;) {
      const uint32_t y = next.fetch_add(1);
      if (y >= y1) break;
      for (uint32_t x = x0; x < x1; x++) {
        for (uint32_t smp = 0; smp < spp; smp++) {
          uint32_t *out = verts + ((size_t)((y - y0) * rw + (x - x0)) * spp + smp) * depth;
          for (uint32_t k = 0; k < depth; k++) out[k] = 0xFFFFFFFFu;
          daxa_u32 s = tea(y * W + x, seed + smp);
          const daxa_f32 jx = rnd(s);
          const daxa_f32 jy = rnd(s);
          const daxa_f32vec2 pixel_center = daxa_f32vec2{glsl_f32(x), glsl_f32(y)} + daxa_f32vec2{jx, jy};
          const daxa_f32vec2 inv_UV = pixel_center / daxa_f32vec2{glsl_f32(W), glsl_f32(H)};
          daxa_f32vec2 d = inv_UV * 2.0f - 1.0f;
          daxa_f32vec4 origin = inv_view * vec4{0, 0, 0, 1};
          vec4 target = inv_proj * vec4{d.x, d.y, 1, 1};
          vec4 direction = inv_view * vec4{normalize(target.xyz()), 0};
          Ray ray = Ray{origin.xyz(), direction.xyz()};
          for (uint32_t k = 0; k < depth; k++) {
            INTERSECT i = intersect(ray);
            if (!i.is_hit) break;
            out[k] = instances[i.instance_hit.instance_id].first_primitive_index + i.instance_hit.primitive_id;
            if (k + 1 == depth) break;
            vec3 o = compute_ray_origin(i.world_hit, i.world_nrm);
            o = compute_ray_origin(o, i.world_nrm);
            vec3 dir = random_cosine_direction(s, i.world_nrm);
            if (normal_near_zero(dir)) dir = i.world_nrm;
            ray = Ray{o, dir};
          }
        }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  return 0;
}

// Known-answer entry points for the shader primitives the kernels reuse.
uint32_t oracle_tea(uint32_t a, uint32_t b) { return tea(a, b); }
float oracle_rnd(uint32_t *seed) { return rnd(*seed); }
void oracle_compute_ray_origin(const float *pos, const float *nrm, float *out) {
  vec3 r = compute_ray_origin(vec3(pos[0], pos[1], pos[2]), vec3(nrm[0], nrm[1], nrm[2]));
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
// intersect_box on a unit-centred box of half extent h (primitives.glsl:273-355)
int oracle_intersect_box(const float *center, float h, const float *o, const float *d, int can_start, int oriented,
                         float *t_out, float *n_out) {
  Box box = Box{vec3(center[0], center[1], center[2]), vec3(h), safeInverse(vec3(h)), mat3(1.f)};
  Ray r = Ray{vec3(o[0], o[1], o[2]), vec3(d[0], d[1], d[2])};
  ct_real t = 0;
  vec3 n;
  bool hit = intersect_box(box, r, t, n, can_start != 0, oriented != 0, safeInverse(r.direction));
  *t_out = t;
  n_out[0] = n.x; n_out[1] = n.y; n_out[2] = n.z;
  return hit ? 1 : 0;
}

}  // extern "C"
