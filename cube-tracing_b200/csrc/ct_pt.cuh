// ct_pt.cuh -- ReSTIR PT: path tracing from the primary hit, path reservoirs,
// the reconnection shift, and temporal / spatial path reuse.  Included by
// ct_kernels.cu after ct_device.cuh.
//
// Semantics follow cube-tracing's shaders with the indirect-illumination
// blocks compiled in (rgen.glsl:271-315, 427-452) and the scene parameters
// rgen.glsl passes to them (no Russian roulette, environment light on, 3
// spatial neighbours in a radius of 1 pixel, defines.glsl:48-63).  The
// shift mapping is SHIFT_MAPPING_RECONNECTION, as rgen.glsl sets it, or,
// with ct_params.pt_shift_mapping = CT_SHIFT_HYBRID, the hybrid shift: the
// base paths choose their reconnection vertex by the shaders' hybrid rule
// (path_check_rc_vertex, path_tracer.glsl:478-516, and the escaped-vertex
// marking of :306-330 and :800-820), and a shift replays the source path's
// random numbers from the destination's primary hit up to the vertex before
// the reconnection vertex, then reconnects (shift_hybrid below).  The
// replay is traced inline; PATH_STATE's replay fields and its accumulated
// radiance L, which only the shaders' replay loop reads, are left out.
//
// One thread per pixel; bounce rays and shadow rays are traced inline with
// the same traversal and hit rules as the rest of the library.

// PATH_STATE.flags bits (defines.glsl:65-77)
#define CT_PF_ACTIVE 0x1u
#define CT_PF_HIT 0x2u
#define CT_PF_LIGHT_SAMPLED_UPPER 0x80u
#define CT_PF_LIGHT_SAMPLED_LOWER 0x100u
#define CT_PF_DIFFUSE_PRIMARY_HIT 0x200u

// OBJECT_HIT (shared.inl)
struct ObjHit {
  uint32_t inst, prim;
  f3 hit;
};
__device__ __forceinline__ ObjHit objhit_none() { return ObjHit{CT_MAX_INSTANCES, CT_MAX_PRIMITIVES, mk3(0.f)}; }
// instance_hit_exists / instance_hit_valid (primitives.glsl:211-214, 542-545)
__device__ __forceinline__ bool objhit_exists(uint32_t inst, uint32_t prim) {
  return inst < CT_MAX_INSTANCES && prim < CT_MAX_PRIMITIVES;
}

// INTERSECT (shared.inl:323-334)
struct Isect {
  bool is_hit;
  float distance;
  f3 world_hit, world_nrm, wo, wi;
  uint32_t inst, prim, material_idx;
  Material mat;
};
// intersect_initiliaze (primitives.glsl:195-209); the material is zero
__device__ __forceinline__ Isect isect_empty() {
  Isect i;
  i.is_hit = false;
  i.distance = 0.f;
  i.world_hit = i.world_nrm = i.wo = i.wi = mk3(0.f);
  i.inst = CT_MAX_INSTANCES;
  i.prim = CT_MAX_PRIMITIVES;
  i.material_idx = CT_MAX_MATERIALS;
  i.mat = Material{};
  return i;
}

// PATH_RESERVOIR (shared.inl:405-423)
struct PathRes {
  float M, weight;
  uint32_t path_flags, rc_random_seed;
  f3 F;
  float light_pdf;
  f3 cached_jacobian;
  uint32_t init_random_seed;
  ObjHit rc_hit;
  f3 rc_wi, rc_irr;
};
__device__ __forceinline__ PathRes load_path_res(const ct_path_reservoir &s) {
  PathRes r;
  r.M = s.M; r.weight = s.weight; r.path_flags = s.path_flags; r.rc_random_seed = s.rc_random_seed;
  r.F = ld3(s.F); r.light_pdf = s.light_pdf; r.cached_jacobian = ld3(s.cached_jacobian);
  r.init_random_seed = s.init_random_seed;
  r.rc_hit = ObjHit{s.rc_vertex_hit.object.instance_id, s.rc_vertex_hit.object.primitive_id, ld3(s.rc_vertex_hit.hit)};
  r.rc_wi = ld3(s.rc_vertex_wi); r.rc_irr = ld3(s.rc_vertex_irradiance);
  return r;
}
__device__ __forceinline__ void store_path_res(ct_path_reservoir &s, const PathRes &r) {
  s.M = r.M; s.weight = r.weight; s.path_flags = r.path_flags; s.rc_random_seed = r.rc_random_seed;
  st3(s.F, r.F); s.light_pdf = r.light_pdf; st3(s.cached_jacobian, r.cached_jacobian);
  s.init_random_seed = r.init_random_seed;
  s.rc_vertex_hit.object.instance_id = r.rc_hit.inst; s.rc_vertex_hit.object.primitive_id = r.rc_hit.prim;
  st3(s.rc_vertex_hit.hit, r.rc_hit.hit);
  st3(s.rc_vertex_wi, r.rc_wi); st3(s.rc_vertex_irradiance, r.rc_irr);
}

// path_flags fields (path_reservoir.glsl:65-148)
__device__ __forceinline__ uint32_t pf_path_length(uint32_t f) { return f & 0xFu; }
__device__ __forceinline__ uint32_t pf_rc_length(uint32_t f) { return (f >> 4) & 0xFu; }
__device__ __forceinline__ bool pf_last_nee(uint32_t f) { return ((f >> 16) & 1u) != 0; }
__device__ __forceinline__ uint32_t pf_light_type(uint32_t f) { return (f >> 18) & 3u; }
__device__ __forceinline__ bool pf_delta(uint32_t f, bool before) { return ((f >> (before ? 20 : 21)) & 1u) != 0; }
__device__ __forceinline__ bool pf_transmission(uint32_t f, bool before) { return ((f >> (before ? 22 : 23)) & 1u) != 0; }
__device__ __forceinline__ uint32_t pf_set_path_length(uint32_t f, uint32_t l) { return (f & ~0xFu) | (l & 0xFu); }
__device__ __forceinline__ uint32_t pf_set_rc_length(uint32_t f, uint32_t l) { return (f & ~0xF0u) | ((l & 0xFu) << 4); }
__device__ __forceinline__ uint32_t pf_set_last_nee(uint32_t f, bool v) { return (f & ~0x10000u) | ((v ? 1u : 0u) << 16); }
__device__ __forceinline__ uint32_t pf_set_light_type(uint32_t f, uint32_t t) { return (f & ~0xC0000u) | ((t & 3u) << 18); }

// path_reservoir_initialise (path_reservoir.glsl:150-163)
__device__ __forceinline__ PathRes path_res_init(uint32_t max_depth) {
  PathRes r;
  r.M = 0.f; r.weight = 0.f;
  r.path_flags = pf_set_rc_length(0u, max_depth);
  r.rc_random_seed = 0u; r.F = mk3(0.f); r.light_pdf = 0.f; r.cached_jacobian = mk3(0.f); r.init_random_seed = 0u;
  r.rc_hit = objhit_none(); r.rc_wi = mk3(0.f); r.rc_irr = mk3(0.f);
  return r;
}

// path_F_to_scalar (path_reservoir.glsl:165-167)
__device__ __forceinline__ float path_scalar(f3 c) { return dot(c, f3{0.299f, 0.587f, 0.114f}); }

// path_reservoir_update (path_reservoir.glsl:183-201)
__device__ __forceinline__ bool path_res_update(PathRes &r, f3 in_F, float p, uint32_t &seed) {
  r.M += 1.0f;
  const float w = path_scalar(in_F) / p;
  if (isnan(w) || w == 0.f) return false;
  r.weight += w;
  if (rnd(seed) * r.weight <= w) {
    r.F = in_F;
    return true;
  }
  return false;
}

__device__ __forceinline__ void path_res_take(PathRes &r, const PathRes &in, f3 in_F) {
  r.path_flags = in.path_flags;
  r.rc_random_seed = in.rc_random_seed;
  r.init_random_seed = in.init_random_seed;
  r.cached_jacobian = in.cached_jacobian;
  r.light_pdf = in.light_pdf;
  r.rc_wi = in.rc_wi;
  r.rc_hit = in.rc_hit;
  r.rc_irr = in.rc_irr;
  r.F = in_F;
}

// path_reservoir_merge (path_reservoir.glsl:203-230)
__device__ __forceinline__ bool path_res_merge(PathRes &r, f3 in_F, float in_jacobian, const PathRes &in, uint32_t &seed,
                                               float mis_weight, bool force_add) {
  const float w = path_scalar(in_F) * in_jacobian * in.M * in.weight * mis_weight;
  r.M += in.M;
  if (isnan(w) || w == 0.f) return false;
  r.weight += w;
  if (force_add || rnd(seed) * r.weight <= w) {
    path_res_take(r, in, in_F);
    return true;
  }
  return false;
}

// path_reservoir_merge_with_resampling_MIS (path_reservoir.glsl:232-260)
__device__ __forceinline__ bool path_res_merge_mis(PathRes &r, f3 in_F, float in_jacobian, const PathRes &in,
                                                   uint32_t &seed, float mis_weight) {
  const float w = path_scalar(in_F) * in_jacobian * in.weight * mis_weight;
  r.M += in.M;
  if (isnan(w) || w == 0.f) return false;
  r.weight += w;
  if (rnd(seed) * r.weight <= w) {
    path_res_take(r, in, in_F);
    return true;
  }
  return false;
}

// path_reservoir_finalize_RIS / _GRIS (path_reservoir.glsl:262-275)
__device__ __forceinline__ void path_res_finalize_ris(PathRes &r) {
  const float p_hat = path_scalar(r.F);
  if (p_hat == 0.f || r.M == 0.f) r.weight = 0.f;
  else r.weight = r.weight / (p_hat * r.M);
}
__device__ __forceinline__ void path_res_finalize_gris(PathRes &r) {
  const float p_hat = path_scalar(r.F);
  if (p_hat == 0.f) r.weight = 0.f;
  else r.weight = r.weight / p_hat;
}

// eval_mis with the power heuristic (light.glsl:166-191)
__device__ __forceinline__ float eval_mis(float nf, float f_pdf, float ng, float g_pdf) {
  const float a = nf * f_pdf, b = ng * g_pdf;
  const float f = a * a, g = b * b;
  return f / (f + g);
}

// scene parameters (SCENE_PARAMS, defines.glsl:90-108) as rgen.glsl fills them
struct PtParams {
  uint32_t light_count;  // point lights (light_config.point_light_count)
  uint32_t max_depth;
  float near_field_distance;  // HALF_VOXEL_EXTENT * 0.5
  float roughness_threshold;  // SPECULAR_ROUGHNESS_THRESHOLD
  uint32_t neighbor_count;
  int32_t neighbor_radius;
  float max_influence;        // MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD_PT
  bool hybrid;                // shift_mapping == SHIFT_MAPPING_HYBRID
};
__device__ __forceinline__ PtParams pt_params(const FrameView &F, const ct_params &P, const DevAccel &A) {
  PtParams p;
  p.light_count = F.light_config.point_light_count;
  p.max_depth = F.max_depth;
  p.near_field_distance = P.pt_near_field_distance > 0.0f ? P.pt_near_field_distance : A.extent * 0.5f * 0.5f;
  p.hybrid = P.pt_shift_mapping == CT_SHIFT_HYBRID;
  p.roughness_threshold = 0.2f;
  p.neighbor_count = P.pt_neighbor_count;
  p.neighbor_radius = (int32_t)P.pt_neighbor_radius;
  p.max_influence = P.pt_max_influence_from_the_past;
  return p;
}

__device__ __forceinline__ uint32_t material_index_of(const FrameView &F, uint32_t inst, uint32_t prim) {
  const uint32_t first = F.instances[inst].first_primitive_index;
  const uint32_t actual = first != 0xFFFFFFFFu ? first + prim : first;
  return F.primitives[actual].material_index;
}

// ---------------------------------------------------------------------------
// scatter directions (rcall_scatter.glsl, prng.glsl)
__device__ __forceinline__ bool normal_near_zero(f3 v) {
  const float s = 1e-8f;
  return fabsf(v.x) < s && fabsf(v.y) < s && fabsf(v.z) < s;
}
__device__ __forceinline__ f3 reflection(f3 v, f3 n) { return v - (2.0f * dot(v, n)) * n; }
__device__ __forceinline__ float length_square(f3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
// random_cosine_direction (prng.glsl:84-106); sin/cos of ct_fpmath.h
__device__ __forceinline__ f3 random_cosine_direction(uint32_t &seed, f3 normal) {
  const float r1 = rnd(seed);
  const float r2 = rnd(seed);
  const float z = sqrtf(1.0f - r2);
  const float phi = 2.0f * 3.1415926535897932384626433832795f * r1;
  const float x = ct_cosf(phi) * sqrtf(r2);
  const float y = ct_sinf(phi) * sqrtf(r2);
  f3 u = fabsf(normal.x) > 0.1f ? f3{0.0f, 1.0f, 0.0f} : f3{1.0f, 0.0f, 0.0f};
  u = normalize(cross(normal, u));
  const f3 v = cross(normal, u);
  return x * u + y * v + z * normal;
}
// reflectance / refraction (prng.glsl:214-227)
__device__ __forceinline__ float reflectance(float cosine, float ref_idx) {
  float r0 = (1.0f - ref_idx) / (1.0f + ref_idx);
  r0 = r0 * r0;
  return r0 + (1.0f - r0) * ct_powf(1.0f - cosine, 5.0f);
}
__device__ __forceinline__ f3 refraction(f3 uv, f3 n, float etai_over_etat) {
  const float cos_theta = gmin(dot(-uv, n), 1.0f);
  const f3 r_out_perp = etai_over_etat * (uv + cos_theta * n);
  const f3 r_out_parallel = -sqrtf(fabsf(1.0f - length_square(r_out_perp))) * n;
  return r_out_parallel + r_out_perp;
}

// The scatter callables (rcall_scatter.glsl:11-86) on the call_scatter
// payload: `kind` selects the callable, the material parameters come from
// MATERIAL[mat_idx]; `hit` and `nrm` are updated as the dielectric callable
// does for rays from inside.  Returns call_scatter.done.
__device__ bool scatter_callable(const FrameView &F, uint32_t kind, uint32_t mat_idx, f3 &hit, f3 &nrm, f3 ray_dir,
                                 uint32_t &seed, uint32_t pixel, f3 &scatter) {
  scatter = mk3(0.f);
  bool done = false;
  switch (kind) {
    case 1u: {  // metal (rcall_scatter.glsl:11-19)
      const Material mat = load_material(F, mat_idx);
      const f3 reflected = reflection(ray_dir, nrm);
      scatter = gmin(mat.roughness, 1.0f) * random_cosine_direction(seed, reflected) + (1.0f - mat.roughness) * reflected;
      done = (dot(scatter, nrm) > 0.0f) ? false : true;
    } break;
    case 2u: {  // dielectric (rcall_scatter.glsl:20-62)
      const Material mat = load_material(F, mat_idx);
      float etai_over_etat = mat.ior;
      if (dielectric_face(hit, nrm, ray_dir)) etai_over_etat = 1.0f / etai_over_etat;
      const float cos_theta = gmin(dot(-ray_dir, nrm), 1.0f);
      const float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
      const bool cannot_refract = etai_over_etat * sin_theta > 1.0f;
      if (cannot_refract || reflectance(cos_theta, etai_over_etat) > rnd(seed)) scatter = reflection(ray_dir, nrm);
      else scatter = refraction(ray_dir, nrm, etai_over_etat);
    } break;
    case 3u: {  // constant medium (rcall_scatter.glsl:64-72)
      scatter = random_unit_vector(seed, pixel);
      if (normal_near_zero(scatter)) scatter = nrm;
    } break;
    default: {  // Lambertian, cosine-weighted (rcall_scatter.glsl:74-86)
      scatter = random_cosine_direction(seed, nrm);
      if (normal_near_zero(scatter)) scatter = nrm;
    } break;
  }
  return done;
}

// generate_scatter_ray (path_tracer.glsl:23-57): the callable is chosen by
// the material INDEX's low byte, as the shader does
__device__ bool generate_scatter_ray(const FrameView &F, Isect &i, uint32_t &seed, uint32_t pixel) {
  f3 hit = i.world_hit, nrm = i.world_nrm, scatter;
  const bool done = scatter_callable(F, i.material_idx & 0xFFu, i.material_idx, hit, nrm, i.wo, seed, pixel, scatter);
  i.world_hit = hit;
  i.world_nrm = nrm;
  i.wi = scatter;
  return !done;
}

// ---------------------------------------------------------------------------
// rays

// load_intersection_data_vertex_position (primitives.glsl:567-616): the
// stored vertex re-derived from its voxel by a box test of the ray from
// `world_pos` towards the stored hit point
// The box is the AABB table's entry at INSTANCE.first_primitive_index + id,
// as is_hit_from_ray reads it (primitives.glsl:412-453): after a scene edit
// an id of the previous frame may lie past the instance's current range
// and still names the table entry left there.  Ids past the table (the
// shader would read out of bounds) give no hit.
__device__ Isect load_vertex(const FrameView &F, const DevAccel &A, const ObjHit &v, f3 world_pos) {
  if (v.inst >= A.n_grids) return isect_empty();
  const DevGrid &g = A.grids[v.inst];
  const uint64_t gi = (uint64_t)F.instances[v.inst].first_primitive_index + v.prim;
  if (gi >= F.obj_count) return isect_empty();
  const f3 dir = v.hit - world_pos;
  const f3 ro = xyz(mul(g.world2obj_inst, mk4(world_pos, 1.0f)));
  const f3 rd = xyz(mul(g.world2obj_inst, mk4(dir, 0.0f)));
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  const ct_aabb &b = F.aabbs[gi];
  const f3 c = (ld3(b.minimum) + ld3(b.maximum)) * 0.5f;
  const BoxHit h = box_test(c, radius, inv_radius, ro, rd, true, false, safe_inverse(rd));
  if (!h.hit) return isect_empty();
  f3 pos = world_pos + dir * h.t;
  const f3 nor = xyz(mul(transpose(g.world2obj_inst), mk4(h.n, 0.0f)));
  pos = offset_twice(pos, nor);
  Isect i;
  i.is_hit = true;
  i.distance = length(world_pos - pos);
  i.world_hit = pos;
  i.world_nrm = nor;
  i.wo = normalize(world_pos - pos);
  i.wi = mk3(0.f);
  i.inst = v.inst;
  i.prim = v.prim;
  i.material_idx = material_index_of(F, v.inst, v.prim);
  i.mat = load_material(F, i.material_idx);
  return i;
}

// is_vertex_visible traced in place; a negative distance leaves nothing to
// test (the shader's query range [0, distance] is empty)
struct VisInline {
  const DevAccel &A;
  uint32_t pixel;
  RayStats &rs;
  __device__ bool operator()(f3 o, f3 d, float dist, uint32_t inst, uint32_t prim, bool check, uint32_t) {
    if (!(dist >= 0.0f)) return true;
    rs.shadow++;
    return vertex_visible(A, o, d, dist, inst, prim, check, pixel, rs);
  }
};

// ---------------------------------------------------------------------------
// path state (path_state.glsl:23-78, path_builder.glsl:9-18)
struct PathBuilder {
  ObjHit rc_hit;
  f3 rc_wi;
  uint32_t cached_random_seed, seed, rc_vertex_length, path_flags;
  f3 cached_jacobian;
};
struct __align__(16) PathState {
  uint32_t max_depth, flags, path_length, bounce_counters;
  f3 origin, dir;
  float pdf;
  ObjHit hit;
  f3 thp, prefix_thp;
  float rr_pdf, prev_scatter_pdf;
  uint32_t seed;
  bool is_last_vertex_rough;
  PathBuilder pb;
  PathRes res;
};
__device__ __forceinline__ bool path_active(const PathState &p) { return (p.flags & CT_PF_ACTIVE) != 0; }
__device__ __forceinline__ void path_terminate(PathState &p) { p.flags &= ~CT_PF_ACTIVE; }
__device__ __forceinline__ f3 path_thp(const PathState &p) { return p.thp * p.prefix_thp; }
__device__ __forceinline__ bool path_finished_bounces(const PathState &p) {
  return (p.bounce_counters & 0xFFu) > p.max_depth;
}
__device__ __forceinline__ void path_set_light_sampled(PathState &p, bool upper, bool lower) {
  p.flags = upper ? (p.flags | CT_PF_LIGHT_SAMPLED_UPPER) : (p.flags & ~CT_PF_LIGHT_SAMPLED_UPPER);
  p.flags = lower ? (p.flags | CT_PF_LIGHT_SAMPLED_LOWER) : (p.flags & ~CT_PF_LIGHT_SAMPLED_LOWER);
}

// path_builder_add_escape_vertex / _add_NEE_vertex (path_builder.glsl:33-111)
__device__ bool builder_add_vertex(PathBuilder &pb, uint32_t path_length, f3 wi, f3 path_weight, f3 postfix_weight,
                                   float rr_pdf, float mis_weight, float light_pdf, uint32_t light_type, PathRes &res,
                                   bool nee) {
  if (path_length < 1) return false;
  const bool is_rc_vertex = path_length == pb.rc_vertex_length;
  if (!path_res_update(res, path_weight, rr_pdf, pb.seed)) return false;
  res.path_flags = pb.path_flags;
  res.path_flags = pf_set_path_length(res.path_flags, path_length);
  res.path_flags = pf_set_rc_length(res.path_flags, pb.rc_vertex_length);
  res.path_flags = pf_set_last_nee(res.path_flags, nee);
  res.rc_irr = postfix_weight;
  res.F = path_weight;
  res.rc_wi = pb.rc_wi;
  res.rc_hit = pb.rc_hit;
  res.cached_jacobian = pb.cached_jacobian;
  res.rc_random_seed = pb.cached_random_seed;
  if (is_rc_vertex) {
    if (nee) {
      res.rc_irr = res.rc_irr * light_pdf / mis_weight;
      res.rc_wi = wi;
    } else {
      res.rc_wi = wi;
      res.rc_irr = res.rc_irr / mis_weight;
    }
  }
  res.light_pdf = light_pdf;
  res.path_flags = pf_set_light_type(res.path_flags, light_type);
  return true;
}

// path_builder_mark_escape_vertex_as_rc_vertex (path_builder.glsl:114-139)
// as the shaders call it: the delta, transmission and specular-bounce events
// they pass are never set by these paths, so the three "before" bits are
// cleared (0x100, 0x400, 0x4000000, as the insert functions clear them,
// path_reservoir.glsl:82-124)
__device__ __forceinline__ void mark_escape_rc_vertex(PathRes &res, uint32_t path_length, const ObjHit &hit,
                                                      float light_pdf, uint32_t light_type, f3 irradiance, f3 wi,
                                                      float prev_scatter_pdf, float geometry_factor) {
  res.path_flags = pf_set_rc_length(res.path_flags, path_length);
  res.rc_hit = hit;
  res.path_flags &= ~0x100u;
  res.path_flags &= ~0x400u;
  res.path_flags &= ~0x4000000u;
  res.light_pdf = light_pdf;
  res.cached_jacobian.x = prev_scatter_pdf;
  res.path_flags = pf_set_light_type(res.path_flags, light_type);
  res.rc_irr = irradiance;
  res.rc_wi = wi;
  res.cached_jacobian.z = geometry_factor;
}

// path_generate_scatter_ray (path_tracer.glsl:59-112)
__device__ bool path_generate_scatter_ray(const FrameView &F, PathState &path, Isect &i, uint32_t pixel) {
  bool valid = generate_scatter_ray(F, i, path.seed, pixel);
  if (valid) {
    f3 weight = evaluate_material(i.mat, i.world_nrm, i.wo, i.wi);
    const float pdf = sample_material_pdf(i.mat, i.world_nrm, i.wo, i.wi);
    weight = weight / pdf;
    path.dir = i.wi;
    if (path.path_length == 0) path.flags |= CT_PF_DIFFUSE_PRIMARY_HIT;
    path.thp = path.thp * weight;
    path.pdf = pdf;
    if (path.path_length == path.pb.rc_vertex_length) path.pb.cached_jacobian.y = pdf;
    path.prev_scatter_pdf = pdf;
    if (pdf <= 0.0f) return false;
    path.bounce_counters += 1u;
    valid = path.thp.x > 0.f || path.thp.y > 0.f || path.thp.z > 0.f;
    if (valid && path.path_length <= path.pb.rc_vertex_length) {
      path.prefix_thp = path.thp;
      path.thp = mk3(1.f);
    }
  }
  return valid;
}

// eval_voxel_pdf (path_tracer.glsl:176-205) and path_evaluate_emissive
// (:207-216)
__device__ __forceinline__ float eval_voxel_pdf(f3 pos, const Isect &i, float extent) {
  const f3 to_light = i.world_hit - pos;
  const float dist_sqr = dot(to_light, to_light);
  if (dist_sqr <= CT_HLF_MIN) return 0.f;
  const f3 L = to_light / sqrtf(dist_sqr);
  const float cos_theta = dot(i.world_nrm, -L);
  if (cos_theta <= 0.f) return 0.f;
  const float side = extent;
  const float area = side * side;
  const float denom = gmax(CT_HLF_MIN, cos_theta * area);
  return dist_sqr / denom;
}

// path_handle_emissive_hit (path_tracer.glsl:258-336), no replay
__device__ void path_handle_emissive_hit(const PtParams &pp, PathState &path, const Isect &i, float extent) {
  float light_pdf = 0.f, mis_weight = 1.f;
  f3 Lr = mk3(0.f);
  if (path.path_length != 0) {
    const float selecting = 1.f / (float)pp.light_count;
    light_pdf = selecting * eval_voxel_pdf(path.origin, i, extent);
    mis_weight = eval_mis(1.f, path.pdf, 1.f, light_pdf);
    Lr = path_thp(path) * i.mat.emission * mis_weight;
  }
  const f3 attenuated = path_thp(path) * i.mat.emission;
  const f3 postfix = path.thp * attenuated * mis_weight;
  const uint32_t len = path.path_length >= 1 ? path.path_length - 1u : 0u;
  const bool selected = builder_add_vertex(path.pb, len, path.dir, Lr, postfix, path.rr_pdf, mis_weight, light_pdf,
                                           CT_LIGHT_CUBE, path.res, false);
  // hybrid shift: an emitter met at path length >= 2 before any
  // reconnection vertex can be one (path_tracer.glsl:306-330)
  if (pp.hybrid && selected && path.path_length >= 2 && path.path_length < path.pb.rc_vertex_length) {
    const bool is_far_field = length(i.world_hit - path.origin) >= pp.near_field_distance;
    if (is_far_field && path.is_last_vertex_rough) {
      const f3 disp = path.origin - i.world_hit;
      float geometry_factor = fabsf(dot(i.world_nrm, i.wo)) / dot(disp, disp);
      if (isnan(geometry_factor)) geometry_factor = 0.f;
      mark_escape_rc_vertex(path.res, path.path_length, path.hit, light_pdf, CT_LIGHT_CUBE, i.mat.emission, mk3(0.f),
                            path.prev_scatter_pdf, geometry_factor);
    }
  }
}

// path_handle_sample_light (path_tracer.glsl:338-433) with
// path_generate_light_sample (:218-255): one point light, no replay.
//
// The light sample's shadow-ray answer reaches only PATH_RESERVOIR.M: the
// sample's weight is zero, because LIGHT_SAMPLER.pdf stays 0 and so does the
// MIS weight eval_mis(1, 0, 1, scatter_pdf), and path_builder_finilize
// (path_builder.glsl:31-34) sets M to 1 when the path ends.  The ray is
// traced all the same (it is part of the shader's work), by whatever `vis`
// provides; nothing after it waits for the answer.
template <class VP>
__device__ void path_handle_sample_light(const FrameView &F, const PtParams &pp, PathState &path, const Isect &i,
                                         bool is_rc_vertex, VP &vis, uint32_t pixel) {
  if (path.path_length == path.pb.rc_vertex_length) path.pb.cached_random_seed = path.seed;
  // path_generate_light_sample
  const uint32_t light_index = gmin(urnd_interval(path.seed, 0u, pp.light_count), pp.light_count - 1u);
  Light light;
  if (pp.light_count > 0u) {
    light = load_light(F.point_lights, light_index);
  } else {  // the shader reads element 0 of an empty buffer; taken as a zero light
    light = Light{};
    light.type = CT_LIGHT_NONE;
  }
  const uint32_t ls_type = light.type;
  float pdf = 1.0f / (float)pp.light_count;
  LightSample s = sample_lights(F, i.world_hit, i.world_nrm, i.inst, i.prim, light, pdf, path.seed, true, true,
                                pixel, vis, 0u);
  const f3 ls_dir = normalize(s.l_pos - i.world_hit);
  f3 ls_Li = s.Le / pdf;
  const float ls_pdf = 0.0f;  // LIGHT_SAMPLER.pdf is never set (path_tracer.glsl:228)
  const bool valid_sample = s.vis;
  path_set_light_sampled(path, true, false);
  if (valid_sample) {
    float mis_weight = 1.f;
    const float scatter_pdf = sample_material_pdf(i.mat, i.world_nrm, i.wo, ls_dir);
    mis_weight = mis_weight * eval_mis(1.f, ls_pdf, 1.f, scatter_pdf);
    ls_Li = ls_Li * mis_weight;
    f3 weight = evaluate_material(i.mat, i.world_nrm, i.wo, ls_dir);
    const f3 Lr = weight * ls_Li * path_thp(path);
    if (is_rc_vertex) weight = mk3(1.f);
    builder_add_vertex(path.pb, path.path_length, ls_dir, Lr, weight * ls_Li * path.thp, path.rr_pdf, mis_weight,
                       ls_pdf, ls_type, path.res, true);
  }
}

// path_handle_hit (path_tracer.glsl:596-719), no replay, no hybrid shift
template <class VP>
__device__ void path_handle_hit(const FrameView &F, const PtParams &pp, PathState &path, Isect &i, float extent, VP &vis,
                                uint32_t pixel) {
  // path_length 1 is never emissive: transmission/delta events do not occur
  const bool compute_emissive = path.path_length != 1;
  if (compute_emissive && (i.mat.emission.x > 0.f || i.mat.emission.y > 0.f || i.mat.emission.z > 0.f))
    path_handle_emissive_hit(pp, path, i, extent);
  if (path_finished_bounces(path)) {
    path_terminate(path);
    return;
  }
  const f3 prev_path_origin = path.origin;
  path.origin = offset_twice(i.world_hit, i.world_nrm);
  const bool is_current_rough = i.mat.roughness > pp.roughness_threshold;
  // path_check_rc_vertex (path_tracer.glsl:478-594): without the hybrid shift
  // the first secondary vertex is the reconnection vertex; with it, the
  // first vertex whose incoming segment is far field and which, with its
  // predecessor, is rough
  bool is_rc_vertex = false;
  bool take = path.path_length == 1;
  if (pp.hybrid) {
    const bool is_far_field = length(path.origin - prev_path_origin) >= pp.near_field_distance;
    take = path.path_length >= 1 && path.path_length < path.pb.rc_vertex_length && is_far_field && is_current_rough &&
           path.is_last_vertex_rough;
  }
  if (take) {
    is_rc_vertex = true;
    path.pb.rc_hit = path.hit;
    path.pb.cached_jacobian.x = path.prev_scatter_pdf;
    const f3 disp = prev_path_origin - i.world_hit;
    path.pb.cached_jacobian.z = fabsf(dot(i.world_nrm, i.wo)) / dot(disp, disp);
    if (isnan(path.pb.cached_jacobian.z)) path.pb.cached_jacobian.z = 0.f;
    path.pb.rc_vertex_length = path.path_length;
  }
  path_set_light_sampled(path, false, false);
  path_handle_sample_light(F, pp, path, i, is_rc_vertex, vis, pixel);
  bool valid = path_generate_scatter_ray(F, path, i, pixel);
  if (path.path_length == path.pb.rc_vertex_length) path.pb.cached_random_seed = path.seed;
  path.pb.rc_wi = path.dir;
  path.is_last_vertex_rough = is_current_rough;
  if (!path_active(path)) return;
  if (path_finished_bounces(path)) valid = false;
  if (!valid) path_terminate(path);
}

// path_handle_miss (path_tracer.glsl:721-809)
__device__ void path_handle_miss(const FrameView &F, const PtParams &pp, PathState &path) {
  const float light_pdf = 0.079577471545947667884441881686255f;  // env_map_sampler_eval_pdf
  const float mis_weight = eval_mis(1.f, path.pdf, 1.f, light_pdf);
  const f3 Le = sky_color(F.time, F.is_afternoon, path.dir);
  const f3 Lr = path_thp(path) * Le * mis_weight;
  const bool selected = builder_add_vertex(path.pb, path.path_length, path.dir, Lr, path.thp * Le * mis_weight,
                                           path.rr_pdf, mis_weight, light_pdf, CT_LIGHT_ENV_MAP, path.res, false);
  // hybrid shift: the escaped vertex as reconnection vertex
  // (path_tracer.glsl:800-820)
  if (pp.hybrid && selected && path.path_length >= 1 && path.path_length + 1u < path.pb.rc_vertex_length &&
      path.is_last_vertex_rough)
    mark_escape_rc_vertex(path.res, path.path_length + 1u, objhit_none(), light_pdf, CT_LIGHT_ENV_MAP, Le, path.dir,
                          path.prev_scatter_pdf, 1.f);
  path_terminate(path);
}

// trace_restir_path_tracing (path_tracer.glsl:854-887) as a wavefront: the
// path starts at the primary hit (path_start), then every bounce ray is
// traced by a persistent walker (closest_walk_*) and the vertex it finds is
// shaded (path_shade) until the path ends (path_finish).

// generate_path (path_state.glsl:197-240) and path_handle_primary_hit
// (path_tracer.glsl:435-462); false when no bounce ray follows
__device__ bool path_start(const FrameView &F, const PtParams &pp, PathState &path, f3 ray_origin, f3 ray_dir, Isect i,
                           uint32_t seed, uint32_t pixel) {
  path.max_depth = pp.max_depth;
  path.flags = CT_PF_ACTIVE | CT_PF_HIT;
  path.path_length = 0;
  path.bounce_counters = 0;
  path.origin = ray_origin;
  path.dir = ray_dir;
  path.pdf = 0.f;
  path.thp = mk3(1.f);
  path.prefix_thp = mk3(1.f);
  path.rr_pdf = 1.f;
  path.prev_scatter_pdf = 1.f;
  path.hit = ObjHit{i.inst, i.prim, i.world_hit};
  path.seed = seed;
  path.pb.seed = seed;
  path.pb.rc_hit = objhit_none();
  path.pb.rc_wi = mk3(0.f);
  path.pb.cached_random_seed = 0u;
  path.pb.rc_vertex_length = pp.max_depth;
  path.pb.path_flags = 0u;
  path.pb.cached_jacobian = mk3(0.f);
  path.res = path_res_init(pp.max_depth);
  path.is_last_vertex_rough = true;
  path.origin = offset_twice(i.world_hit, i.world_nrm);
  path_set_light_sampled(path, false, false);
  path.res.init_random_seed = path.seed;
  const bool valid = path_generate_scatter_ray(F, path, i, pixel);
  if (path.path_length == path.pb.rc_vertex_length) path.pb.cached_random_seed = path.seed;
  path.pb.rc_wi = path.dir;
  return valid;
}

// path_finalize / path_output (path_tracer.glsl:811-852)
__device__ __forceinline__ void path_finish(PathState &path) {
  path.flags &= ~CT_PF_ACTIVE;
  path.res.M = 1.0f;
  path_res_finalize_ris(path.res);
}

// The vertex a bounce ray found, as intersect() returns it (bounce.glsl:9-125):
// the ray query walks candidates by the box test of is_hit_from_ray on the ray
// with its origin moved by compute_ray_origin(origin, direction) (rays may
// start inside a box) and commits the first hit with t in [0, MAX_DISTANCE];
// the hit position and normal are the ones is_hit_from_ray returns for that
// voxel (primitives.glsl:412-453), the distance is measured from the
// unmoved origin.
// bounce_geometry: the hit point and normal alone.
__device__ __forceinline__ void bounce_geometry(const DevAccel &A, f3 ray_origin, f3 ray_dir, uint32_t inst,
                                                uint32_t prim, uint32_t gprim, f3 &pos, f3 &nrm) {
  const f3 key_o = compute_ray_origin(ray_origin, ray_dir);
  const DevGrid &g = A.grids[inst];
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  const f3 ro = xyz(mul(g.world2obj_inst, mk4(key_o, 1.0f)));
  const f3 rd = xyz(mul(g.world2obj_inst, mk4(ray_dir, 0.0f)));
  const uint32_t pk = __ldg(&A.voxel_coord[gprim]);
  const f3 c = voxel_center(A, g, (int)(pk & 0x3FFu), (int)((pk >> 10) & 0x3FFu), (int)((pk >> 20) & 0x3FFu), prim);
  const BoxHit h = box_test(c, radius, inv_radius, ro, rd, true, false, safe_inverse(rd));
  pos = key_o + ray_dir * h.t;
  nrm = xyz(mul(transpose(g.world2obj_inst), mk4(h.n, 0.0f)));
}
__device__ Isect bounce_vertex(const FrameView &F, const DevAccel &A, f3 ray_origin, f3 ray_dir, uint32_t inst,
                               uint32_t prim, uint32_t gprim) {
  Isect i;
  i.is_hit = true;
  bounce_geometry(A, ray_origin, ray_dir, inst, prim, gprim, i.world_hit, i.world_nrm);
  i.inst = inst;
  i.prim = prim;
  i.material_idx = material_index_of(F, inst, prim);
  i.mat = load_material(F, i.material_idx);
  i.distance = length(ray_origin - i.world_hit);
  i.wo = normalize(ray_origin - i.world_hit);
  i.wi = mk3(0.f);
  return i;
}

// one step of the path loop after its bounce ray (path_next_vertex and
// path_handle_hit / path_handle_miss, path_tracer.glsl:114-126, 866-879)
template <class VP>
__device__ void path_shade(const FrameView &F, const DevAccel &A, const PtParams &pp, PathState &path, bool hit,
                           uint32_t inst, uint32_t prim, uint32_t gprim, VP &vis, uint32_t pixel) {
  if (hit) {
    Isect i = bounce_vertex(F, A, path.origin, path.dir, inst, prim, gprim);
    path.hit = ObjHit{i.inst, i.prim, i.world_hit};
    path.flags |= CT_PF_HIT;
    path.path_length++;
    path_handle_hit(F, pp, path, i, A.extent, vis, pixel);
  } else {
    path.flags &= ~CT_PF_HIT;
    path_handle_miss(F, pp, path);
  }
}

// Closest hit of a bounce ray as a resumable walk (the walker refills lanes
// whose ray is done): intersect()'s candidate test and commit rule
// (QueryVisitor, closest mode) over every instance in turn.  Where the
// instance's object-space ray lives is the caller's choice (Store):
//  * ObjRay: held, with its reciprocal, in memory the caller places (shared
//    memory in the bounce walker), so that a box test reads it;
//  * NoObjRay: held nowhere, derived again from the world ray at every box
//    test (for one-thread-per-ray walks, where registers are what bounds
//    occupancy).
struct ClosestWalk {
  uint32_t inst;     // instance being walked
  DdaState dda;
  HitRecord best;
};
struct NoObjRay {};
// the object-space ray of instance g, derived from the world ray `ray`
template <class RayFn>
struct ObjRayDerived {
  const RayFn &ray;
  const DevGrid &g;
  __device__ void operator()(f3 &ro, f3 &rd) const {
    f3 o, d;
    ray(o, d);
    const f3 key_o = compute_ray_origin(o, d);
    ro = xyz(mul(g.world2obj_inst, mk4(key_o, 1.0f)));
    rd = xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
  }
  __device__ f3 inv(f3 rd) const { return safe_inverse(rd); }
};
// The world-space ray is not kept in the walk (the walkers are register
// bound): `ray(o, d)` gives the bounce ray back when the walk moves to
// another instance, and the query origin is derived from it again.
template <class RayFn, class Store>
__device__ __forceinline__ bool closest_walk_instance(const DevAccel &A, ClosestWalk &w, const RayFn &ray, Store &R) {
  for (; w.inst < A.n_grids; w.inst++) {
    const DevGrid &g = A.grids[w.inst];
    f3 ro, rd;
    ObjRayDerived<RayFn>{ray, g}(ro, rd);
    if (dda_init(A, g, ro, rd, 0.f, w.best.hit ? w.best.t : 1e9f, w.dda)) {
      if constexpr (std::is_same<Store, ObjRay>::value) {
        R.ro = ro;
        R.rd = rd;
        R.ird = safe_inverse(rd);
      }
      return true;
    }
  }
  return false;
}
// true when the ray is already decided (no instance to walk)
template <class Store>
__device__ __forceinline__ bool closest_walk_begin(const DevAccel &A, ClosestWalk &w, f3 origin, f3 dir, Store &R) {
  w.best = HitRecord{false, 0.f, 0u, 0u, 0u};
  w.inst = 0;
  return !closest_walk_instance(A, w, [&](f3 &o, f3 &d) { o = origin; d = dir; }, R);
}
template <class RayFn, class Store>
__device__ __forceinline__ int closest_walk_advance(const DevAccel &A, ClosestWalk &w, int budget, uint32_t pixel,
                                                    RayStats &rs, const RayFn &ray, Store &R) {
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  const DevGrid &g = A.grids[w.inst];
  int st;
  if constexpr (std::is_same<Store, ObjRay>::value) {
    QueryVisitor<ObjRayRef> v{A, g, ObjRayRef{R}, radius, inv_radius, true, 1e9f, w.inst, false, INFINITY,
                              0xFFFFFFFFu, false, 0u, 0u, w.best, 0u};
    st = dda_run(A, g, w.dda, v, rs, budget);
    rs.voxel_tests += v.tests;
  } else {
    QueryVisitor<ObjRayDerived<RayFn>> v{A, g, ObjRayDerived<RayFn>{ray, g}, radius, inv_radius, true, 1e9f,
                                         w.inst, false, INFINITY, 0xFFFFFFFFu, false, 0u, 0u, w.best, 0u};
    st = dda_run(A, g, w.dda, v, rs, budget);
    rs.voxel_tests += v.tests;
  }
  if (st == DDA_LIMIT) ct_latch_error(CT_ERR_ITER_LIMIT, 4, pixel);
  if (st == DDA_MORE) return DDA_MORE;
  w.inst++;
  return closest_walk_instance(A, w, ray, R) ? DDA_MORE : DDA_DONE;
}

// intersect() (bounce.glsl:9-125) run to the end in place
__device__ Isect intersect_closest(const FrameView &F, const DevAccel &A, f3 origin, f3 dir, uint32_t pixel,
                                   RayStats &rs) {
  ClosestWalk w;
  NoObjRay R;
  rs.bounce++;
  const auto ray = [&](f3 &o, f3 &d) { o = origin; d = dir; };
  if (!closest_walk_begin(A, w, origin, dir, R))
    while (closest_walk_advance(A, w, 1 << 20, pixel, rs, ray, R) == DDA_MORE) {
    }
  if (!w.best.hit) return isect_empty();
  rs.bounce_hits++;
  return bounce_vertex(F, A, origin, dir, w.best.inst, w.best.prim, w.best.gprim);
}

// Records the one shadow ray a call site asks for, answering "visible"; for
// rays whose answer nothing reads (the light sample above), which the caller
// queues for the shadow-ray walker afterwards.
struct VisRecord {
  bool has;
  float4 a, b;
  uint2 c;
  __device__ bool operator()(f3 o, f3 d, float dist, uint32_t inst, uint32_t prim, bool check, uint32_t) {
    if (!(dist >= 0.0f)) return true;  // empty query range: nothing to trace
    has = true;
    a = make_float4(o.x, o.y, o.z, dist);
    b = make_float4(d.x, d.y, d.z, 0.f);
    c = make_uint2(inst | (check ? 0x80000000u : 0u), prim);
    return true;
  }
};

// ---------------------------------------------------------------------------
// reconnection shift (compute_shifted_integrand_reconnection, shift.glsl:25-350):
// the integrand of `s`'s path moved to the vertex `dst` (the primary hit, or
// with the hybrid shift the replayed vertex before the reconnection vertex),
// and its Jacobian.  Visibility of the reconnection segment is traced when
// `eval_visibility`.  use_hybrid_shift: the reconnection vertex is at the
// path's own reconnection length and the segment to it must be far field;
// use_cached_jacobian: the source side's pdfs and geometry term come from
// s.cached_jacobian, which a successful shift replaces with the destination's.
template <class VP>
__device__ f3 shift_reconnection(const FrameView &F, const DevAccel &A, float &dst_jacobian, Isect dst, Isect src,
                                 PathRes &s, bool eval_visibility, VP &vis, uint32_t slot, bool use_hybrid_shift = false,
                                 bool use_cached_jacobian = false, float near_field_distance = 0.f) {
  dst_jacobian = 0.f;
  if (s.weight == 0.f) return mk3(0.f);  // compute_shifted_integrand_ (shift.glsl:452-455)
  const uint32_t rc_vertex_length = use_hybrid_shift ? pf_rc_length(s.path_flags) : 1u;
  const bool rc_exists = objhit_exists(s.rc_hit.inst, s.rc_hit.prim);
  const uint32_t path_length = pf_path_length(s.path_flags);
  const bool is_last_nee = pf_last_nee(s.path_flags);
  const bool is_transmission = pf_transmission(s.path_flags, true);
  // compute_new_ray_origin (primitives.glsl:259-264)
  const f3 sn = is_transmission ? -src.world_nrm : src.world_nrm;
  src.world_hit = offset_twice(src.world_hit, sn);
  const f3 dn = is_transmission ? -dst.world_nrm : dst.world_nrm;
  dst.world_hit = offset_twice(dst.world_hit, dn);
  if (!rc_exists) {
    // environment reconnection: the stored light type keeps two bits and
    // never equals GEOMETRY_LIGHT_ENV_MAP (5), so the shader's branch
    // (shift.glsl:68-109) is never taken
    return mk3(0.f);
  }
  const bool is_rc_final = path_length == rc_vertex_length;
  const bool is_rc_escaped = path_length + 1u == rc_vertex_length && !is_last_nee;
  const bool is_rc_nee = is_rc_final && is_last_nee;
  if (pf_delta(s.path_flags, true) || pf_delta(s.path_flags, false)) return mk3(0.f);
  const Isect rc = load_vertex(F, A, s.rc_hit, dst.world_hit);
  const f3 dst_connection_v = -rc.wo;
  const f3 src_connection_v = normalize(rc.world_hit - src.world_hit);
  const f3 shifted_disp = rc.world_hit - dst.world_hit;
  const float shifted_dist2 = dot(shifted_disp, shifted_disp);
  const float shifted_cosine = fabsf(dot(rc.world_nrm, -dst_connection_v));
  if (use_hybrid_shift && !(sqrtf(shifted_dist2) >= near_field_distance)) return mk3(0.f);
  f3 dst_cached = mk3(0.f);
  dst_cached.z = shifted_cosine / shifted_dist2;
  float jacobian;
  if (use_cached_jacobian) {
    jacobian = dst_cached.z / s.cached_jacobian.z;
  } else {
    const f3 original_disp = rc.world_hit - src.world_hit;
    const float original_dist2 = dot(original_disp, original_disp);
    const float original_cosine = fabsf(dot(rc.world_nrm, -src_connection_v));
    jacobian = dst_cached.z * original_dist2 / original_cosine;
  }
  auto invalid = [](float j) { return j <= 0.f || isnan(j) || isinf(j); };
  if (invalid(jacobian)) return mk3(0.f);
  const float dst_pdf1 = sample_material_pdf(dst.mat, dst.world_nrm, dst.wo, dst_connection_v);
  const float dst_pdf1_all = dst_pdf1;
  dst_cached.x = dst_pdf1;
  const float src_pdf1 = use_cached_jacobian ? s.cached_jacobian.x
                                             : sample_material_pdf(src.mat, src.world_nrm, src.wo, src_connection_v);
  jacobian = jacobian * (dst_pdf1 / src_pdf1);
  if (invalid(jacobian)) return mk3(0.f);
  const f3 dst_f1 = evaluate_material(dst.mat, dst.world_nrm, dst.wo, dst_connection_v);
  float dst_rc_pdf_all = 0.f, dst_pdf2 = 1.f, dst_rc_pdf = 1.f, src_rc_pdf = 1.f;
  if (!is_rc_escaped) {
    dst_rc_pdf = sample_material_pdf(rc.mat, rc.world_nrm, rc.wo, s.rc_wi);
    dst_rc_pdf_all = dst_rc_pdf;
    dst_cached.y = dst_rc_pdf;
    src_rc_pdf = use_cached_jacobian ? s.cached_jacobian.y
                                     : sample_material_pdf(rc.mat, rc.world_nrm, -src_connection_v, s.rc_wi);
    dst_pdf2 = !is_rc_nee ? dst_rc_pdf : s.light_pdf;
  }
  f3 dst_f2 = mk3(1.0f);
  if (!is_rc_escaped) dst_f2 = evaluate_material(rc.mat, rc.world_nrm, rc.wo, s.rc_wi);
  if ((dst_f1.x == 0.f && dst_f1.y == 0.f && dst_f1.z == 0.f) || (dst_f2.x == 0.f && dst_f2.y == 0.f && dst_f2.z == 0.f))
    return mk3(0.f);
  const f3 dst_integrand_no_f1 = dst_f2 / dst_pdf2 * s.rc_irr;
  f3 dst_integrand = dst_f1 / dst_pdf1 * dst_integrand_no_f1;
  if (is_rc_escaped) dst_integrand = dst_integrand * eval_mis(1.f, dst_pdf1_all, 1.f, s.light_pdf);
  if (is_rc_final) {
    if (pf_light_type(s.path_flags) != 4u) {  // GEOMETRY_LIGHT_ANALITIC
      const float lp = s.light_pdf;
      const float m = eval_mis(1.f, is_rc_nee ? lp : dst_rc_pdf_all, 1.f, is_rc_nee ? dst_rc_pdf_all : lp);
      dst_integrand = dst_integrand * m;
      if (!is_rc_nee) jacobian = jacobian * (dst_rc_pdf / src_rc_pdf);
    }
  }
  if (!is_rc_final && !is_rc_escaped) jacobian = jacobian * (dst_rc_pdf / src_rc_pdf);
  if (invalid(jacobian)) return mk3(0.f);
  if (eval_visibility) {
    const f3 dir = normalize(rc.world_hit - dst.world_hit);
    const float dist = length(dst.world_hit - rc.world_hit);
    if (!vis(dst.world_hit, dir, dist, rc.inst, rc.prim, true, slot)) return mk3(0.f);
  }
  if (any_nan_inf(dst_integrand)) return mk3(0.f);
  dst_jacobian = jacobian;
  if (use_cached_jacobian) s.cached_jacobian = dst_cached;
  return dst_integrand;
}

// The hybrid shift's random-number replay (the role of
// trace_random_replay_path_hybrid_simple, path_tracer.glsl:889-958): from
// the destination's primary hit `dst`, the source path's scatter random
// numbers (its init_random_seed, one light-sample draw skipped at every
// vertex the base path sampled a light at) are replayed up to vertex
// rc_length - 1, whose intersection and throughput prefix it returns.  The
// shift is not invertible, and the replay fails, when a replayed vertex
// before that one would itself have been the offset path's reconnection
// vertex (far-field incoming segment, rough, rough predecessor) or when
// vertex rc_length - 1 is not rough (path_check_rc_vertex, :517-590), or
// when the replay misses the scene or meets a zero throughput.
__device__ bool replay_prefix(const FrameView &F, const DevAccel &A, const PtParams &pp, const Isect &dst,
                              const PathRes &src, uint32_t rc_length, Isect &prev, f3 &tp, uint32_t pixel,
                              RayStats &rs) {
  uint32_t seed = src.init_random_seed;
  Isect i = dst;
  f3 origin = offset_twice(i.world_hit, i.world_nrm);
  // the scatter at the primary hit (path_generate_scatter_ray, path length 0)
  if (!generate_scatter_ray(F, i, seed, pixel)) return false;
  f3 weight = evaluate_material(i.mat, i.world_nrm, i.wo, i.wi);
  float pdf = sample_material_pdf(i.mat, i.world_nrm, i.wo, i.wi);
  weight = weight / pdf;
  if (pdf <= 0.0f) return false;
  f3 thp = weight;
  if (!(thp.x > 0.f || thp.y > 0.f || thp.z > 0.f)) return false;
  f3 dir = i.wi;
  bool last_rough = true;  // the base path's value at its first bounce
  for (uint32_t len = 1; len < rc_length; len++) {
    Isect h = intersect_closest(F, A, origin, dir, pixel, rs);
    if (!h.is_hit) return false;
    const f3 new_origin = offset_twice(h.world_hit, h.world_nrm);
    const bool is_far_field = length(new_origin - origin) >= pp.near_field_distance;
    const bool rough = h.mat.roughness > pp.roughness_threshold;
    if (is_far_field && rough && last_rough) return false;  // would reconnect here: not invertible
    if (len + 1u == rc_length) {
      if (!rough) return false;
      prev = h;
      tp = thp;
      return true;
    }
    rnd(seed);  // the light sample the base path drew at this vertex
    if (!generate_scatter_ray(F, h, seed, pixel)) return false;
    weight = evaluate_material(h.mat, h.world_nrm, h.wo, h.wi);
    pdf = sample_material_pdf(h.mat, h.world_nrm, h.wo, h.wi);
    weight = weight / pdf;
    if (pdf <= 0.0f) return false;
    thp = thp * weight;
    if (!(thp.x > 0.f || thp.y > 0.f || thp.z > 0.f)) return false;
    origin = new_origin;
    dir = h.wi;
    last_rough = rough;
  }
  return false;
}

// Where shift_hybrid gets a replay from: traced here and now, or (temporal
// reuse) read from the results k_pt_replay left for the pixel.
struct InlineReplay {
  const FrameView &F;
  const DevAccel &A;
  const PtParams &pp;
  uint32_t pixel;
  RayStats &rs;
  __device__ bool operator()(const Isect &dst, const PathRes &src, uint32_t rc_length, Isect &prev, f3 &tp) const {
    return replay_prefix(F, A, pp, dst, src, rc_length, prev, tp, pixel, rs);
  }
};

// The hybrid shift (compute_shifted_integrand_hybrid, shift.glsl:352-444,
// as the method defines it): a path whose reconnection vertex is vertex 1
// reconnects from the destination's primary hit; a longer prefix is
// replayed first and reconnects from its last vertex, with the source
// side's pdfs and geometry term taken from its cached Jacobian.  The
// integrand is the replayed prefix throughput times the reconnection's,
// and the Jacobian the reconnection's (the replay is the identity on
// random numbers).  A path without a reconnection vertex does not shift.
template <class VP, class RP>
__device__ f3 shift_hybrid(const FrameView &F, const DevAccel &A, const PtParams &pp, float &dst_jacobian,
                           const Isect &dst, const Isect &src, PathRes &temp, bool eval_visibility, VP &vis,
                           uint32_t slot, const RP &replay) {
  dst_jacobian = 0.f;
  if (temp.weight == 0.f) return mk3(0.f);
  const uint32_t rc_length = pf_rc_length(temp.path_flags);
  const uint32_t path_length = pf_path_length(temp.path_flags);
  const bool escaped = path_length + 1u == rc_length;
  if (!(rc_length <= path_length || escaped) || !objhit_exists(temp.rc_hit.inst, temp.rc_hit.prim)) return mk3(0.f);
  Isect prev = dst;
  f3 tp = mk3(1.f);
  if (rc_length > 1u && !replay(dst, temp, rc_length, prev, tp)) return mk3(0.f);
  PathRes s = temp;
  float jac = 0.f;
  const f3 rc_tp = shift_reconnection(F, A, jac, prev, src, s, eval_visibility, vis, slot, true, rc_length > 1u,
                                      pp.near_field_distance);
  dst_jacobian = jac;
  temp.cached_jacobian = s.cached_jacobian;
  return tp * rc_tp;
}

// compute_shifted_integrand_ (shift.glsl:446-490): the shift the scene
// parameters select, on `temp` (whose cached Jacobian the hybrid shift may
// replace)
// (HYBRID is the kernels' compile-time copy of pp.hybrid, so that the
// reconnection-only kernels carry none of the replay's registers)
template <bool HYBRID, class VP, class RP>
__device__ f3 shift_path(const FrameView &F, const DevAccel &A, const PtParams &pp, float &dst_jacobian,
                         const Isect &dst, const Isect &src, PathRes &temp, bool eval_visibility, VP &vis,
                         uint32_t slot, const RP &replay) {
  if constexpr (HYBRID)
    return shift_hybrid(F, A, pp, dst_jacobian, dst, src, temp, eval_visibility, vis, slot, replay);
  else
    return shift_reconnection(F, A, dst_jacobian, dst, src, temp, eval_visibility, vis, slot);
}

// shift_and_merge_reservoir (shift.glsl:504-531) with force_merge
template <bool HYBRID, class VP, class RP>
__device__ bool shift_and_merge(const FrameView &F, const DevAccel &A, const PtParams &pp, float &dst_jacobian,
                                const Isect &dst_i, PathRes &dst, const Isect &src_i, const PathRes &src,
                                uint32_t &seed, VP &vis, uint32_t slot, const RP &replay) {
  PathRes temp = src;
  const f3 integrand = shift_path<HYBRID>(F, A, pp, dst_jacobian, dst_i, src_i, temp, true, vis, slot, replay);
  const bool selected = path_res_merge(dst, integrand, dst_jacobian, temp, seed, 1.f, true);
  if (!selected) dst.F = mk3(0.f);
  dst.M = src.M;
  dst.weight = src.weight;
  return selected;
}
