// ct_device.cuh -- device-side scene access, voxel traversal and the
// direct-lighting building blocks shared by the frame kernels.  Included by
// exactly one translation unit (ct_kernels.cu), which owns the device
// status word.
//
// Semantics follow cube-tracing's shaders (file:line given per function);
// the data layout, traversal and thread mapping are this library's own.
#pragma once
#include <cstdint>
#include "ct_types.cuh"
#include "ct_fpmath.h"

// device error word: [0] status, [1] detail, [2] pixel
__device__ uint32_t g_ct_error[4];
__device__ __forceinline__ void ct_latch_error(uint32_t status, uint32_t detail, uint32_t pixel) {
  if (atomicCAS(&g_ct_error[0], 0u, status) == 0u) {
    g_ct_error[1] = detail;
    g_ct_error[2] = pixel;
  }
}

// Work counters (flushed to ct_params.counters_address when
// CT_PARAM_COUNT_RAYS is set): rays by kind, 8^3 bricks the walks entered,
// voxel box tests, light candidates evaluated, neighbour records read by
// spatial reuse, temporal reuse records read, shaded (hit) pixels.
struct RayStats {
  uint32_t primary, shadow, bounce, bricks, voxel_tests, candidates, neighbours, temporal, hits, bounce_hits,
      walker_bricks;
};

// ---------------------------------------------------------------------------
// per-frame view of the caller's buffers (WORLD / RESTIR / Status tables)
struct FrameView {
  uint32_t W, H;
  const ct_instance *instances;
  const ct_instance *instances_prev;
  const ct_primitive *primitives;
  const ct_aabb *aabbs;
  const uint32_t *remap_p;    // WORLD.remapped_primitive_address (CT_REMAP_BIT)
  const uint32_t *remap_l;    // WORLD.remapped_cube_light_address
  const ct_material *materials;
  const ct_light *point_lights;
  const ct_light *cube_lights;
  const ct_light *env_lights;
  ct_reservoir *prev_reservoir;
  ct_reservoir *int_reservoir;
  ct_reservoir *cur_reservoir;
  ct_di_info *prev_di;
  ct_di_info *di;
  ct_velocity *velocity;
  ct_path_reservoir *out_path_reservoir;
  ct_path_reservoir *temporal_path_reservoir;
  float *indirect_color;
  float4 *swapchain;
  const float4 *previous_swapchain;
  float4 *taa_frame;
  ct_light_config light_config;
  uint32_t frame_number, is_active, obj_count, is_afternoon, max_depth;
  float time;
  const ct_camera_view *camera;
};

__device__ __forceinline__ f3 ld3(const float *p) { return f3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(float *p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

struct Material {
  uint32_t type;
  f3 diffuse, specular, emission;
  float roughness, ior;
};
__device__ __forceinline__ Material load_material(const FrameView &F, uint32_t idx) {
  const ct_material &m = F.materials[idx];
  Material r;
  r.type = m.type;
  r.diffuse = ld3(m.diffuse);
  r.specular = ld3(m.specular);
  r.emission = ld3(m.emission);
  r.roughness = m.roughness;
  r.ior = m.ior;
  return r;
}

struct Light {
  f3 position, emissive;
  uint32_t inst, prim;
  float size;
  uint32_t type;
};
__device__ __forceinline__ Light load_light(const ct_light *buf, uint32_t idx) {
  const ct_light &l = buf[idx];
  Light r;
  r.position = ld3(l.position);
  r.emissive = ld3(l.emissive);
  r.inst = l.instance_info.instance_id;
  r.prim = l.instance_info.primitive_id;
  r.size = l.size;
  r.type = l.type;
  return r;
}
// light_get_by_type (light.glsl:47-64); unknown types give an empty light
__device__ __forceinline__ Light light_get_by_type(const FrameView &F, uint32_t type, uint32_t idx) {
  if (type == CT_LIGHT_POINT) return load_light(F.point_lights, idx);
  if (type == CT_LIGHT_ENV_MAP) return load_light(F.env_lights, idx);
  if (type == CT_LIGHT_CUBE) return load_light(F.cube_lights, idx);
  Light l = {};
  l.type = CT_LIGHT_NONE;
  return l;
}

// ---------------------------------------------------------------------------
// sky / environment (mat.glsl:111-202, light.glsl:71-76)
__device__ __forceinline__ f3 bg_mix(f3 dir, f3 a, f3 b) {
  f3 u = normalize(dir);
  float t = 0.5f * (u.y + 1.0f);
  return gmix(a, b, t);
}
__device__ __forceinline__ f3 bg_day(f3 d) { return bg_mix(d, mk3(1.0f, 1.0f, 1.0f), mk3(0.5f, 0.7f, 1.0f)); }
__device__ __forceinline__ f3 bg_night(f3 d) { return bg_mix(d, mk3(0.2f, 0.2f, 0.3f), mk3(0.2f, 0.2f, 0.5f)); }
__device__ __forceinline__ f3 bg_sunset(f3 d) { return bg_mix(d, mk3(0.8f, 0.4f, 0.0f), mk3(1.0f, 0.4f, 0.0f)); }
__device__ __forceinline__ f3 bg_sunrise(f3 d) { return bg_mix(d, mk3(0.7f, 0.35f, 0.0f), mk3(0.8f, 0.4f, 0.0f)); }
__device__ __forceinline__ f3 sky_color(float t, uint32_t is_afternoon, f3 dir) {
  const float night_duration = 0.5f, sunrise_duration = 0.10f, full_daylight_transition = 0.10f,
              full_night_transition = 0.10f;
  const float sunrise_end = night_duration + sunrise_duration;
  const float sunrise_to_daylight = sunrise_end + full_daylight_transition;
  const float zenith_transition = 1.0f - sunrise_to_daylight;
  const float daylight_end = 1.0f - zenith_transition;
  const float sunset_start = 1.0f - zenith_transition - sunrise_duration;
  const float sunset_end = 1.0f - zenith_transition - sunrise_duration - full_night_transition;
  if (is_afternoon) {
    if (t < night_duration) return bg_night(dir);
    if (t < sunrise_end) return gmix(bg_night(dir), bg_sunrise(dir), t);
    if (t < sunrise_to_daylight) return gmix(bg_sunrise(dir), bg_sunset(dir), t);
    return gmix(bg_sunset(dir), bg_day(dir), t);
  }
  if (t > daylight_end) return gmix(bg_sunrise(dir), bg_day(dir), t);
  if (t > sunset_start) return gmix(bg_sunset(dir), bg_sunrise(dir), t);
  if (t > sunset_end) return gmix(bg_night(dir), bg_sunset(dir), t);
  return bg_night(dir);
}

// ---------------------------------------------------------------------------
// voxel lookup
__device__ __forceinline__ uint32_t table_entry(const DevAccel &A, const DevGrid &g, int bx, int by, int bz) {
  if ((unsigned)bx >= (unsigned)g.bdim[0] || (unsigned)by >= (unsigned)g.bdim[1] || (unsigned)bz >= (unsigned)g.bdim[2])
    return CT_EMPTY_SLOT;
  return __ldg(&A.brick_table[g.table_offset + ((uint32_t)bz * g.bdim[1] + by) * g.bdim[0] + bx]);
}
// primitive id (instance relative) of grid-local voxel (x,y,z), or -1
__device__ __forceinline__ uint32_t cell_index(const DevGrid &g, int bx, int by, int bz) {
  return g.table_offset + ((uint32_t)bz * g.bdim[1] + by) * g.bdim[0] + bx;
}
__device__ __forceinline__ int32_t voxel_prim(const DevAccel &A, const DevGrid &g, int x, int y, int z) {
  const int bx = x >> 3, by = y >> 3, bz = z >> 3;
  uint32_t e = table_entry(A, g, bx, by, bz);
  if (!(e & CT_NEAR_BIT)) return -1;
  uint32_t slot = e & CT_EMPTY_SLOT;
  uint32_t local = (uint32_t)(x & 7) + 8u * (uint32_t)(y & 7) + 64u * (uint32_t)(z & 7);
  uint32_t w = __ldg(&A.brick_mask[slot * CT_MASK_WORDS + (local >> 5)]);
  if (!((w >> (local & 31u)) & 1u)) return -1;
  uint32_t ps = __ldg(&A.brick_pslot[cell_index(g, bx, by, bz)]);
  return (int32_t)__ldg(&A.brick_prim[ps * 512u + local]);
}

// voxel centre in object space: (AABB.minimum + AABB.maximum) * 0.5
// (primitives.glsl:369, 397, 439, 524)
__device__ __forceinline__ f3 voxel_center(const DevAccel &A, const DevGrid &g, int x, int y, int z, uint32_t prim) {
  if (g.grid_exact) {
    float e = A.extent;
    f3 mn = f3{(float)(x + g.gmin[0]) * e, (float)(y + g.gmin[1]) * e, (float)(z + g.gmin[2]) * e};
    f3 mx = f3{(float)(x + g.gmin[0] + 1) * e, (float)(y + g.gmin[1] + 1) * e, (float)(z + g.gmin[2] + 1) * e};
    return (mn + mx) * 0.5f;
  }
  const ct_aabb &b = A.aabbs[g.first_primitive_index + prim];
  return (ld3(b.minimum) + ld3(b.maximum)) * 0.5f;
}

// ---------------------------------------------------------------------------
// DDA over one instance's brick map, offering every voxel whose box the ray
// passes within `eps` voxels of.  The box test (and therefore which voxel is
// hit and at what distance) is rounding-sensitive near voxel edges; visiting
// this superset of candidates makes the result depend only on the box test
// itself, never on the traversal order or on how the DDA rounds.
//
// Visitor interface:
//   bool visit(int x, int y, int z, uint32_t prim)   returns true to stop
//   float stop_t()                                    cells entered later are skipped
struct DdaRay {
  f3 o, d;       // grid-local voxel units (origin relative to the grid's first voxel)
  f3 inv;        // 1/d (inf for zero components)
  float eps;
};

template <class V>
__device__ bool dda_visit_cell(const DevAccel &A, const DevGrid &g, int x, int y, int z, V &vis) {
  int32_t pr = voxel_prim(A, g, x, y, z);
  if (pr < 0) return false;
  vis.tests++;
  return vis.visit(x, y, z, (uint32_t)pr);
}

// t interval over which the ray lies within eps of the plane coordinate c on
// axis a, clipped to [t0, t1]
__device__ __forceinline__ void near_interval(float o, float d, float inv, float c, float eps, float t0, float t1,
                                              float &lo, float &hi) {
  if (d == 0.f) {
    if (fabsf(o - c) < eps) { lo = t0; hi = t1; } else { lo = 1.f; hi = 0.f; }
    return;
  }
  float ta = (c - eps - o) * inv, tb = (c + eps - o) * inv;
  lo = fmaxf(fminf(ta, tb), t0);
  hi = fminf(fmaxf(ta, tb), t1);
}

// Neighbours of cell c that the ray passes within eps of while it crosses c
// (t in [t_in, t_out]), except the previous and the next cell of the walk,
// as a mask over the 3x3x3 block (bit (dz+1)*9 + (dy+1)*3 + (dx+1)); the walk
// visits them in increasing bit order.  A pure function of its arguments, out
// of line: the walk calls it only after dda_near_faces found the ray close to
// a face.
__device__ __noinline__ uint32_t dda_neighbour_mask(DdaRay r, int c0, int c1, int c2, float t_in, float t_out,
                                                    int entry_axis, int exit_axis, int s0, int s1, int s2) {
  const int c[3] = {c0, c1, c2}, step[3] = {s0, s1, s2};
  const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z}, inv[3] = {r.inv.x, r.inv.y, r.inv.z};
  // near-face intervals: [axis][0 = lower face, 1 = upper face]
  float lo[3][2], hi[3][2];
  bool any_other = false;
#pragma unroll
  for (int a = 0; a < 3; a++) {
#pragma unroll
    for (int f = 0; f < 2; f++) {
      near_interval(o[a], d[a], inv[a], (float)(c[a] + f), r.eps, t_in, t_out, lo[a][f], hi[a][f]);
      bool is_entry = (a == entry_axis) && (f == (step[a] > 0 ? 0 : 1));
      bool is_exit = (a == exit_axis) && (f == (step[a] > 0 ? 1 : 0));
      if (!is_entry && !is_exit && lo[a][f] <= hi[a][f]) any_other = true;
    }
  }
  if (!any_other) {
    // only the corner between the entry and exit faces can be near
    if (entry_axis < 0 || entry_axis == exit_axis) return 0u;
    int fe = step[entry_axis] > 0 ? 0 : 1, fx = step[exit_axis] > 0 ? 1 : 0;
    float l = fmaxf(lo[entry_axis][fe], lo[exit_axis][fx]), h = fminf(hi[entry_axis][fe], hi[exit_axis][fx]);
    if (l > h) return 0u;
    int n[3] = {0, 0, 0};
    n[entry_axis] -= step[entry_axis];
    n[exit_axis] += step[exit_axis];
    return 1u << ((n[2] + 1) * 9 + (n[1] + 1) * 3 + (n[0] + 1));
  }
  // general case: every neighbour whose touching faces are all near at a
  // common time, except the previous and the next cell of the walk
  uint32_t mask = 0u;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int dd[3] = {dx, dy, dz};
        if (dx == 0 && dy == 0 && dz == 0) continue;
        int nz = (dx != 0) + (dy != 0) + (dz != 0);
        if (nz == 1) {
          int a = dx != 0 ? 0 : (dy != 0 ? 1 : 2);
          if (a == entry_axis && dd[a] == -step[a]) continue;
          if (a == exit_axis && dd[a] == step[a]) continue;
        }
        float l = t_in, h = t_out;
#pragma unroll
        for (int a = 0; a < 3; a++) {
          if (dd[a] == 0) continue;
          int f = dd[a] > 0 ? 1 : 0;
          l = fmaxf(l, lo[a][f]);
          h = fminf(h, hi[a][f]);
        }
        if (l > h) continue;
        mask |= 1u << ((dz + 1) * 9 + (dy + 1) * 3 + (dx + 1));
      }
  return mask;
}

// Cheap screen for dda_neighbour_mask, on a box of cells [lo, hi]: false
// only when the ray stays well clear (2 eps + 1e-3 voxels) of every face of
// the box other than its entry and exit faces, and crosses the box too far
// from the entry/exit edge to pass near it.  The segment does not cross
// those other faces' planes, so its distance to each is smallest at an end
// point.  A voxel outside the box that the ray passes within eps of, while
// inside the box, lies beyond one of these faces: none when this is false.
__device__ __forceinline__ bool dda_near_box(const DdaRay &r, const int lo[3], const int hi[3], float t_in, float t_out,
                                             int entry_axis, int exit_axis, const int step[3]) {
  const float m = 2.0f * r.eps + 1e-3f;
  const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
  bool near = false;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float p0 = o[a] + d[a] * t_in, p1 = o[a] + d[a] * t_out;
    const float dlo = fminf(p0, p1) - (float)lo[a], dhi = (float)(hi[a] + 1) - fmaxf(p0, p1);
    const bool lo_excl = (a == entry_axis && step[a] > 0) || (a == exit_axis && step[a] < 0);
    const bool hi_excl = (a == entry_axis && step[a] < 0) || (a == exit_axis && step[a] > 0);
    near = near || (!lo_excl && !(dlo >= m)) || (!hi_excl && !(dhi >= m));
  }
  if (near) return true;
  if (entry_axis >= 0 && entry_axis != exit_axis) {
    const float inv[3] = {r.inv.x, r.inv.y, r.inv.z};
    float ie = 0.f, ix = 0.f;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (a == entry_axis) ie = fabsf(inv[a]);
      if (a == exit_axis) ix = fabsf(inv[a]);
    }
    if (!(t_out - t_in > (r.eps + m) * (ie + ix))) return true;
  }
  return false;
}
// the same screen on the single cell c
__device__ __forceinline__ bool dda_near_faces(const DdaRay &r, const int c[3], float t_in, float t_out, int entry_axis,
                                               int exit_axis, const int step[3]) {
  return dda_near_box(r, c, c, t_in, t_out, entry_axis, exit_axis, step);
}

// Walk state, resumable: dda_run advances it by a bounded number of cells so
// that a warp can refill lanes whose walk has ended (k_trace_shadow).  Kept
// in named scalars so that a walk lives in registers.
struct DdaState {
  DdaRay r;
  int cx, cy, cz;  // current cell
  float t_in, t1;
  int entry_axis;
  int cur_bkey;
  uint32_t cur_ent;
  int steps;
};

__device__ __forceinline__ int ct_step_of(float d) { return d > 0.f ? 1 : (d < 0.f ? -1 : 0); }

// false: the ray does not overlap the grid within [tmin, tmax]
__device__ __forceinline__ bool dda_init(const DevAccel &A, const DevGrid &g, f3 o_obj, f3 d_obj, float tmin,
                                         float tmax, DdaState &s) {
  const float e = A.extent;
  DdaRay &r = s.r;
  // x / e is x * (1 / e) exactly when e is a power of two (the usual voxel
  // edges 1 and 2^-5), and one multiply is far cheaper than an IEEE division
  if ((__float_as_uint(e) & 0x007FFFFFu) == 0u && e > 1e-30f && e < 1e30f) {
    const float ie = 1.0f / e;
    r.o = f3{o_obj.x * ie - (float)g.gmin[0], o_obj.y * ie - (float)g.gmin[1], o_obj.z * ie - (float)g.gmin[2]};
    r.d = f3{d_obj.x * ie, d_obj.y * ie, d_obj.z * ie};
  } else {
    r.o = f3{o_obj.x / e - (float)g.gmin[0], o_obj.y / e - (float)g.gmin[1], o_obj.z / e - (float)g.gmin[2]};
    r.d = f3{d_obj.x / e, d_obj.y / e, d_obj.z / e};
  }
  r.inv = f3{1.f / r.d.x, 1.f / r.d.y, 1.f / r.d.z};
  const float G[3] = {(float)(g.bdim[0] * CT_BRICK), (float)(g.bdim[1] * CT_BRICK), (float)(g.bdim[2] * CT_BRICK)};
  const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z}, inv[3] = {r.inv.x, r.inv.y, r.inv.z};
  float t0 = tmin, t1 = tmax;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (d[a] == 0.f) {
      if (o[a] < 0.f || o[a] > G[a]) return false;
    } else {
      float ta = (0.f - o[a]) * inv[a], tb = (G[a] - o[a]) * inv[a];
      t0 = fmaxf(t0, fminf(ta, tb));
      t1 = fminf(t1, fmaxf(ta, tb));
    }
  }
  if (!(t0 <= t1)) return false;
  // rounding allowance of the box test (see the comment above)
  float L = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float g0 = (float)g.gmin[a];
    L = fmaxf(L, fmaxf(fabsf(o[a] + g0), fabsf(o[a] + g0 + d[a] * t1)));
  }
  r.eps = 2e-4f + 4e-6f * L;
  int cc[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float p = __fmaf_rn(d[a], t0, o[a]);
    int ci = (int)floorf(p);
    int gi = g.bdim[a] * CT_BRICK;
    cc[a] = ci < 0 ? 0 : (ci >= gi ? gi - 1 : ci);
  }
  s.cx = cc[0]; s.cy = cc[1]; s.cz = cc[2];
  s.t_in = t0;
  s.t1 = t1;
  s.entry_axis = -1;
  s.cur_bkey = -1;
  s.cur_ent = 0;
  // the walk's cap: CT_DDA_MAX_STEPS counts from here, so a smaller
  // A.max_steps (a test's) ends the walk after that many cells
  s.steps = CT_DDA_MAX_STEPS - (int)A.max_steps;
  return true;
}

enum { DDA_DONE = 0, DDA_MORE = 1, DDA_LIMIT = 2 };

// leaving the box [lo, hi] (cells) along one axis
__device__ __forceinline__ void ct_box_exit(int a, int st, int lo, int hi, float o, float inv, float &tb, int &ax) {
  if (st == 0) return;
  const float tt = ((float)(st > 0 ? hi + 1 : lo) - o) * inv;
  if (tt < tb) { tb = tt; ax = a; }
}
// the cell after leaving the box at tb: across the exit face on the exit
// axis, the ray's cell clamped to the box on the others
__device__ __forceinline__ int ct_box_next(bool exit_axis, int st, int lo, int hi, float d, float tb, float o) {
  if (exit_axis) return st > 0 ? hi + 1 : lo - 1;
  const int ci = (int)floorf(__fmaf_rn(d, tb, o));
  return ci < lo ? lo : (ci > hi ? hi : ci);
}

// Advances the walk by at most `budget` steps.  Every step leaves one
// axis-aligned box of cells through its exit face: a brick that is not NEAR
// (no voxel in or next to it: nothing to test), a cube of cells with no
// occupied cell that has the current cell as its corner and extends in the
// ray's directions (the brick's octant field, see DevAccel), taken when the
// ray stays clear of the cube's side faces (so that no voxel beside the cube
// comes within eps of the ray inside it), or a single cell: an occupied one,
// or the current one when the ray passes near a side face of its cube.  A
// single cell's voxel is tested, and its neighbours when the ray passes
// within eps of their faces.  DDA_DONE: the walk ended (left the grid,
// passed stop_t, or the visitor stopped it).
//
// ct_ray_octant: the field of the ray's octant (an axis the ray does not
// move along counts as increasing); cell_field: the field's edge k at cell
// (x, y, z); ct_box_axis: the box on one axis, the cube of edge k from cell
// c towards the ray's direction, clipped to the grid's `cells`.
__device__ __forceinline__ uint32_t ct_ray_octant(int sx, int sy, int sz) {
  return (sx < 0 ? 1u : 0u) | (sy < 0 ? 2u : 0u) | (sz < 0 ? 4u : 0u);
}
__device__ __forceinline__ int cell_field(const DevAccel &A, const DevGrid &g, uint32_t octant, int x, int y, int z) {
  // a grid has at most 1024^3 cells (10-bit voxel coordinates), so the words
  // of its 8 octants (one per 8 cells each) index in 32 bits
  const uint32_t Y = (uint32_t)g.bdim[1] * CT_BRICK, Z = (uint32_t)g.bdim[2] * CT_BRICK;
  const uint32_t w = ((octant * Z + (uint32_t)z) * Y + (uint32_t)y) * (uint32_t)g.bdim[0] + ((uint32_t)x >> 3);
  return ct_field_edge((__ldg(A.cell_field + g.field_offset + w) >> ((x & 7) * 4)) & 15u);
}
__device__ __forceinline__ void ct_box_axis(int c, int st, int k, int cells, int &lo, int &hi) {
  const int e = k > 0 ? k - 1 : 0;
  if (st < 0) {
    lo = max(c - e, 0);
    hi = c;
  } else {
    lo = c;
    hi = min(c + e, cells - 1);
  }
}

// A box (the occupied-free cube from the cell field) is taken whole only when
// the ray stays clear of its side faces (dda_near_box); otherwise the step
// is the current cell alone.  Returns true when the step is a single cell
// whose voxel and near neighbours must be tested: an occupied cell (k == 0)
// or a fallback cell.  Updates the box and its exit.
__device__ __forceinline__ bool ct_screen_box(const DdaRay &r, int k, int cx, int cy, int cz, int sx, int sy, int sz,
                                              float t_in, int entry_axis, int &lox, int &hix, int &loy, int &hiy,
                                              int &loz, int &hiz, float &tb, int &ax) {
  if (k == 0) return true;
  const int lo3[3] = {lox, loy, loz}, hi3[3] = {hix, hiy, hiz}, st3[3] = {sx, sy, sz};
  if (!dda_near_box(r, lo3, hi3, t_in, tb, entry_axis, ax, st3)) return false;
  lox = hix = cx;
  loy = hiy = cy;
  loz = hiz = cz;
  tb = INFINITY;
  ax = 0;
  ct_box_exit(0, sx, lox, hix, r.o.x, r.inv.x, tb, ax);
  ct_box_exit(1, sy, loy, hiy, r.o.y, r.inv.y, tb, ax);
  ct_box_exit(2, sz, loz, hiz, r.o.z, r.inv.z, tb, ax);
  return true;
}

template <class V>
__device__ __forceinline__ int dda_run(const DevAccel &A, const DevGrid &g, DdaState &s, V &vis, RayStats &rs,
                                       int budget) {
  const DdaRay &r = s.r;
  const int sx = ct_step_of(r.d.x), sy = ct_step_of(r.d.y), sz = ct_step_of(r.d.z);
  const uint32_t octant = ct_ray_octant(sx, sy, sz);
  const int gx = g.bdim[0] * CT_BRICK, gy = g.bdim[1] * CT_BRICK, gz = g.bdim[2] * CT_BRICK;
  int cx = s.cx, cy = s.cy, cz = s.cz;
  float t_in = s.t_in;
  int entry_axis = s.entry_axis;
  int result = DDA_MORE;
  for (int it = 0; it < budget; it++) {
    if (++s.steps > CT_DDA_MAX_STEPS) { result = DDA_LIMIT; break; }
    const int bkey = (cx >> 3) | ((cy >> 3) << 10) | ((cz >> 3) << 20);  // bricks per axis < 1024
    if (bkey != s.cur_bkey) {
      rs.bricks++;
      s.cur_bkey = bkey;
    }
    const int k = cell_field(A, g, octant, cx, cy, cz);
    int lox, hix, loy, hiy, loz, hiz;
    ct_box_axis(cx, sx, k, gx, lox, hix);
    ct_box_axis(cy, sy, k, gy, loy, hiy);
    ct_box_axis(cz, sz, k, gz, loz, hiz);
    float tb = INFINITY;
    int ax = 0;
    ct_box_exit(0, sx, lox, hix, r.o.x, r.inv.x, tb, ax);
    ct_box_exit(1, sy, loy, hiy, r.o.y, r.inv.y, tb, ax);
    ct_box_exit(2, sz, loz, hiz, r.o.z, r.inv.z, tb, ax);
    if (ct_screen_box(r, k, cx, cy, cz, sx, sy, sz, t_in, entry_axis, lox, hix, loy, hiy, loz, hiz, tb, ax)) {
      // a single cell: its voxel, then the neighbours the ray passes near
      if (k == 0) {
        const int32_t pr = voxel_prim(A, g, cx, cy, cz);
        if (pr >= 0) {
          vis.tests++;
          if (vis.visit(cx, cy, cz, (uint32_t)pr)) { result = DDA_DONE; break; }
        }
      }
      const int c3[3] = {cx, cy, cz}, st3[3] = {sx, sy, sz};
      if (dda_near_faces(r, c3, t_in, tb, entry_axis, ax, st3)) {
        bool stop = false;
        for (uint32_t m = dda_neighbour_mask(r, cx, cy, cz, t_in, tb, entry_axis, ax, sx, sy, sz); m; m &= m - 1u) {
          const int nb = __ffs(m) - 1;
          if (dda_visit_cell(A, g, cx + nb % 3 - 1, cy + (nb / 3) % 3 - 1, cz + nb / 9 - 1, vis)) {
            stop = true;
            break;
          }
        }
        if (stop) { result = DDA_DONE; break; }
      }
    }
    // The next box begins at tb, computed in grid-local coordinates whose
    // rounding (a few ulps of the coordinate scale L, with r.eps = 2e-4 +
    // 4e-6 L) is amplified by |1/d| on the exit axis: a voxel behind that
    // face has box-test distance at least tb - 1e-6 L |1/d|.  The walk ends
    // only when that bound lies past the stop distance, so that a voxel on
    // the same face plane as the best hit (an exact tie) is still seen.
    const float st = vis.stop_t();
    const float slack = ((r.eps - 2e-4f) * 0.25f + 1e-6f) * fabsf(ax == 0 ? r.inv.x : (ax == 1 ? r.inv.y : r.inv.z));
    if (tb - slack > st + 1e-5f * fabsf(st) + 1e-6f || tb - slack >= s.t1) { result = DDA_DONE; break; }
    cx = ct_box_next(ax == 0, sx, lox, hix, r.d.x, tb, r.o.x);
    cy = ct_box_next(ax == 1, sy, loy, hiy, r.d.y, tb, r.o.y);
    cz = ct_box_next(ax == 2, sz, loz, hiz, r.d.z, tb, r.o.z);
    const bool out = ax == 0 ? (cx < 0 || cx >= gx) : (ax == 1 ? (cy < 0 || cy >= gy) : (cz < 0 || cz >= gz));
    if (out) { result = DDA_DONE; break; }
    t_in = tb;
    entry_axis = ax;
  }
  s.cx = cx; s.cy = cy; s.cz = cz;
  s.t_in = t_in;
  s.entry_axis = entry_axis;
  return result;
}

// Returns false if the walk hit its step cap (error latched by the caller).
template <class V>
__device__ bool dda_traverse(const DevAccel &A, const DevGrid &g, f3 o_obj, f3 d_obj, float tmin, float tmax, V &vis,
                             RayStats &rs) {
  DdaState s;
  if (!dda_init(A, g, o_obj, d_obj, tmin, tmax, s)) return true;
  return dda_run(A, g, s, vis, rs, CT_DDA_MAX_STEPS + 1) != DDA_LIMIT;
}

// ---------------------------------------------------------------------------
// Hit rules
//
// closest hit by box-test distance, ties -> lowest global primitive index.
struct HitRecord {
  bool hit;
  float t;
  uint32_t inst, prim, gprim;
};
__device__ __forceinline__ bool hit_better(float t, uint32_t g, const HitRecord &b) {
  return !b.hit || t < b.t || (t == b.t && g < b.gprim);
}

// Intersection shader semantics (rint.glsl:10-43 with
// is_hit_from_ray_providing_model, primitives.glsl:357-382): object-space ray
// from the instance's TLAS transform, oriented box test (division), rays may
// start inside a box, hits reported for t > 0 within [tmin, current tmax].
struct PrimaryVisitor {
  const DevAccel &A; const DevGrid &g;
  f3 ro, rd, inv_rd;  // object space
  f3 radius, inv_radius;
  float tmin, tmax;
  uint32_t inst;
  HitRecord &best;
  uint32_t tests;
  __device__ float stop_t() const { return best.hit ? best.t : tmax; }
  __device__ bool visit(int x, int y, int z, uint32_t prim) {
    f3 c = voxel_center(A, g, x, y, z, prim);
    BoxHit h = box_test(c, radius, inv_radius, ro, rd, true, true, inv_rd);
    float t = h.hit ? h.t : -1.0f;
    if (!(t > 0.f)) return false;
    float cur = best.hit ? best.t : tmax;
    if (!(t >= tmin && t <= cur)) return false;
    uint32_t gp = g.first_primitive_index + prim;
    if (hit_better(t, gp, best)) { best.hit = true; best.t = t; best.inst = inst; best.prim = prim; best.gprim = gp; }
    return false;
  }
};

// Ray-query semantics (light.glsl:106-137, bounce.glsl:85-119): candidates
// are tested with is_hit_from_ray (primitives.glsl:412-453): object-space ray
// from the inverse of INSTANCE.transform, non-oriented box test
// (multiplication by safeInverse(direction)).  Visibility: the first hit in
// (t, primitive) order with t in [0, t_max] decides; it blocks unless it is
// the light's own voxel.  Closest query: the first such hit is the result.
// The object-space ray and its reciprocal are asked of `ray` at every box
// test: a FixedRay, or an ObjRayRef to a ray held elsewhere.
struct FixedRay {
  f3 ro, rd;
  __device__ void operator()(f3 &o, f3 &d) const { o = ro; d = rd; }
  __device__ f3 inv(f3 d) const { return safe_inverse(d); }
};
// a walk's object-space ray and the reciprocal direction the box test takes,
// held once (in shared memory by the bounce walker) instead of derived again
// at every box test
struct ObjRay {
  f3 ro, rd, ird;
};
struct ObjRayRef {
  const ObjRay &R;
  __device__ void operator()(f3 &o, f3 &d) const { o = R.ro; d = R.rd; }
  __device__ f3 inv(f3) const { return R.ird; }
};
template <class RayObj>
struct QueryVisitor {
  const DevAccel &A; const DevGrid &g;
  RayObj ray;  // object space
  f3 radius, inv_radius;
  bool can_start;
  float tmax;
  uint32_t inst;
  // visibility mode: decisive key of the target
  bool visibility;
  float target_t; uint32_t target_g; bool has_target; uint32_t target_inst, target_prim;
  HitRecord &best;  // closest mode result / visibility: blocking hit
  uint32_t tests;
  __device__ float stop_t() const {
    if (visibility) return fminf(tmax, target_t);
    return best.hit ? best.t : tmax;
  }
  __device__ bool visit(int x, int y, int z, uint32_t prim) {
    if (visibility && has_target && inst == target_inst && prim == target_prim) return false;
    f3 c = voxel_center(A, g, x, y, z, prim);
    f3 ro, rd;
    ray(ro, rd);
    BoxHit h = box_test(c, radius, inv_radius, ro, rd, can_start, false, ray.inv(rd));
    if (!h.hit) return false;
    float t = h.t;
    if (!(t >= 0.f && t <= tmax)) return false;
    uint32_t gp = g.first_primitive_index + prim;
    if (visibility) {
      if (t < target_t || (t == target_t && gp < target_g)) {
        best.hit = true; best.t = t; best.inst = inst; best.prim = prim; best.gprim = gp;
        return true;  // blocked
      }
      return false;
    }
    if (t <= (best.hit ? best.t : tmax) && hit_better(t, gp, best)) {
      best.hit = true; best.t = t; best.inst = inst; best.prim = prim; best.gprim = gp;
    }
    return false;
  }
};



__device__ __forceinline__ f3 half_extent_v(const DevAccel &A) { float h = A.extent * 0.5f; return f3{h, h, h}; }

// closest hit of a camera ray (traceRayEXT with the RIS_SELECTION hit group)
__device__ HitRecord trace_primary(const DevAccel &A, f3 o, f3 d, float tmin, float tmax, uint32_t pixel,
                                   RayStats &rs) {
  HitRecord best = {false, 0.f, 0u, 0u, 0u};
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  for (uint32_t i = 0; i < A.n_grids; i++) {
    const DevGrid &g = A.grids[i];
    f3 ro = xyz(mul(g.world2obj_tlas, mk4(o, 1.0f)));
    f3 rd = xyz(mul(g.world2obj_tlas, mk4(d, 0.0f)));
    PrimaryVisitor v{A, g, ro, rd, safe_inverse(rd), radius, inv_radius, tmin, tmax, i, best, 0u};
    if (!dda_traverse(A, g, ro, rd, tmin, best.hit ? best.t : tmax, v, rs)) ct_latch_error(CT_ERR_ITER_LIMIT, 1, pixel);
    rs.voxel_tests += v.tests;
  }
  return best;
}

// is_vertex_visible (light.glsl:82-142) under the visibility rule above.
__device__ bool vertex_visible(const DevAccel &A, f3 o, f3 d, float distance, uint32_t t_inst, uint32_t t_prim,
                               bool check_instance, uint32_t pixel, RayStats &rs) {
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  // key of the target voxel (the decisive order is (t, global primitive))
  float target_t = INFINITY;
  uint32_t target_g = 0xFFFFFFFFu;
  bool has_target = check_instance && t_inst < A.n_grids;
  if (has_target) {
    const DevGrid &g = A.grids[t_inst];
    if (t_prim < g.primitive_count) {
      uint32_t gp = g.first_primitive_index + t_prim;
      uint32_t pk = __ldg(&A.voxel_coord[gp]);
      int x = (int)(pk & 0x3FFu), y = (int)((pk >> 10) & 0x3FFu), z = (int)((pk >> 20) & 0x3FFu);
      f3 ro = xyz(mul(g.world2obj_inst, mk4(o, 1.0f)));
      f3 rd = xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
      f3 c = voxel_center(A, g, x, y, z, t_prim);
      BoxHit h = box_test(c, radius, inv_radius, ro, rd, false, false, safe_inverse(rd));
      if (h.hit && h.t >= 0.f && h.t <= distance) { target_t = h.t; target_g = gp; }
    }
  }
  for (uint32_t i = 0; i < A.n_grids; i++) {
    const DevGrid &g = A.grids[i];
    f3 ro = xyz(mul(g.world2obj_inst, mk4(o, 1.0f)));
    f3 rd = xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
    HitRecord blk = {false, 0.f, 0u, 0u, 0u};
    QueryVisitor<FixedRay> v{A, g, FixedRay{ro, rd}, radius, inv_radius, false, distance, i, true, target_t,
                             target_g, has_target, t_inst, t_prim, blk, 0u};
    float tlim = fminf(distance, target_t);
    if (!dda_traverse(A, g, ro, rd, 0.f, tlim, v, rs)) ct_latch_error(CT_ERR_ITER_LIMIT, 2, pixel);
    rs.voxel_tests += v.tests;
    if (blk.hit) return false;
  }
  return true;
}

// is_vertex_visible with previous_frame set (light.glsl:82-142 over
// p.tlas_previous), for temporal reuse after a scene edit.  Candidates come
// from the previous scene's brick map `A`: a primitive is a candidate when
// its voxel box in that scene passes the query's box test with t in
// [0, distance] -- the boxes a BVH over the previous AABBs reports.  The
// intersection shader then tests the CURRENT AABB of the same (instance,
// primitive) id: is_hit_from_ray (primitives.glsl:412-453) reads
// WORLD.aabb_address and, with previous_frame set, the current INSTANCE.
// The first candidate in (t, primitive) order decides, as in vertex_visible.
// Needs exact voxel grids in `A` (the previous boxes are recomputed from
// their integer coordinates).
struct PrevQueryVisitor {
  const DevAccel &A; const DevGrid &g;
  const ct_aabb *aabbs;
  uint32_t cur_first;
  f3 ro, rd, inv_rd;
  f3 radius, inv_radius;
  float tmax;
  uint32_t inst;
  float target_t; uint32_t target_g; bool has_target; uint32_t target_inst, target_prim;
  bool blocked;
  uint32_t tests;
  __device__ float stop_t() const { return tmax; }
  __device__ bool visit(int x, int y, int z, uint32_t prim) {
    if (has_target && inst == target_inst && prim == target_prim) return false;
    const BoxHit h0 = box_test(voxel_center(A, g, x, y, z, prim), radius, inv_radius, ro, rd, false, false, inv_rd);
    if (!h0.hit || !(h0.t >= 0.f && h0.t <= tmax)) return false;
    const ct_aabb &b = aabbs[cur_first + prim];
    const BoxHit h = box_test((ld3(b.minimum) + ld3(b.maximum)) * 0.5f, radius, inv_radius, ro, rd, false, false, inv_rd);
    if (!h.hit || !(h.t >= 0.f && h.t <= tmax)) return false;
    const uint32_t gp = g.first_primitive_index + prim;
    if (h.t < target_t || (h.t == target_t && gp < target_g)) {
      blocked = true;
      return true;
    }
    return false;
  }
};

__device__ bool vertex_visible_prev(const DevAccel &A, const FrameView &F, f3 o, f3 d, float distance,
                                    uint32_t t_inst, uint32_t t_prim, bool check_instance, uint32_t pixel,
                                    RayStats &rs) {
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  for (uint32_t i = 0; i < A.n_grids; i++)
    if (!A.grids[i].grid_exact) {
      ct_latch_error(CT_ERR_UNSUPPORTED, 41, pixel);
      return true;
    }
  float target_t = INFINITY;
  uint32_t target_g = 0xFFFFFFFFu;
  const bool has_target = check_instance && t_inst < A.n_grids;
  if (has_target) {
    const DevGrid &g = A.grids[t_inst];
    if (t_prim < g.primitive_count) {
      const uint32_t gp = g.first_primitive_index + t_prim;
      const uint32_t pk = __ldg(&A.voxel_coord[gp]);
      const int x = (int)(pk & 0x3FFu), y = (int)((pk >> 10) & 0x3FFu), z = (int)((pk >> 20) & 0x3FFu);
      const f3 ro = xyz(mul(g.world2obj_inst, mk4(o, 1.0f)));
      const f3 rd = xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
      const f3 inv_rd = safe_inverse(rd);
      const BoxHit h0 = box_test(voxel_center(A, g, x, y, z, t_prim), radius, inv_radius, ro, rd, false, false, inv_rd);
      if (h0.hit && h0.t >= 0.f && h0.t <= distance) {
        const ct_aabb &b = F.aabbs[F.instances[t_inst].first_primitive_index + t_prim];
        const BoxHit h =
            box_test((ld3(b.minimum) + ld3(b.maximum)) * 0.5f, radius, inv_radius, ro, rd, false, false, inv_rd);
        if (h.hit && h.t >= 0.f && h.t <= distance) { target_t = h.t; target_g = gp; }
      }
    }
  }
  for (uint32_t i = 0; i < A.n_grids; i++) {
    const DevGrid &g = A.grids[i];
    const f3 ro = xyz(mul(g.world2obj_inst, mk4(o, 1.0f)));
    const f3 rd = xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
    PrevQueryVisitor v{A, g, F.aabbs, F.instances[i].first_primitive_index, ro, rd, safe_inverse(rd), radius,
                       inv_radius, distance, i, target_t, target_g, has_target, t_inst, t_prim, false, 0u};
    if (!dda_traverse(A, g, ro, rd, 0.f, distance, v, rs)) ct_latch_error(CT_ERR_ITER_LIMIT, 3, pixel);
    rs.voxel_tests += v.tests;
    if (v.blocked) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// vertex_visible split for k_trace_shadow into a stepping phase and a testing
// phase.  A visibility query's decision does not depend on the order in which
// candidates are tested: the stop distance is fixed (min(distance, target
// t)), and the ray is blocked when ANY candidate voxel other than the target
// passes the box test with t in [0, distance] and a key below the target's.
// So a lane may step on past a dilated cell and leave that cell's tests (its
// own voxel and the neighbours the ray passes within eps of, exactly the
// candidates dda_run offers) to a job that the warp tests later, 32 jobs at a
// time, one per lane.  The stepping phase keeps only the cheap part of a
// dilated cell (its occupancy bit and the near-face screen, which rule out
// nearly all of them); the box tests and neighbour masks, rare and long, run
// with full warps instead of one lane at a time.  A lane may enumerate a few
// cells past its first blocker; the decision is the same.

// a lane's ray as both phases read it, kept in shared memory
struct ShadowRay {
  DdaRay r;               // grid-local, as dda_init made it
  f3 ro, rd, ird;         // object space, and safe_inverse(rd) as the box test takes it
  float tmax;             // the query distance
  float target_t;         // key of the target voxel (INFINITY: none)
  uint32_t target_g;
  uint32_t target_inst;   // 0xFFFFFFFF when the query does not check an instance
  uint32_t target_prim;
  uint32_t inst;          // instance being walked
};

// The ray's object-space form for instance `inst`, then dda_init over that
// instance's grid (false: no overlap).  `known`: the caller already has the
// object-space origin `kro`, direction `krd` and safe_inverse(krd) `kird`
// for this instance (the target test's), which are used as they are.
__device__ __forceinline__ bool shadow_ray_instance(const DevAccel &A, ShadowRay &R, DdaState &s, uint32_t inst, f3 o,
                                                    f3 d, bool known = false, f3 kro = f3{}, f3 krd = f3{},
                                                    f3 kird = f3{}) {
  const DevGrid &g = A.grids[inst];
  const f3 ro = known ? kro : xyz(mul(g.world2obj_inst, mk4(o, 1.0f)));
  const f3 rd = known ? krd : xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
  if (!dda_init(A, g, ro, rd, 0.f, fminf(R.tmax, R.target_t), s)) return false;
  R.r = s.r;
  R.ro = ro;
  R.rd = rd;
  if (known) {
    R.ird = kird;
  } else if (A.extent == 1.0f) {
    // with a voxel edge of 1 the walk's direction is rd itself (rd * 1), so
    // its reciprocals are safe_inverse's wherever rd is not 0
    R.ird = f3{rd.x == 0.0f ? 1e12f : s.r.inv.x, rd.y == 0.0f ? 1e12f : s.r.inv.y,
               rd.z == 0.0f ? 1e12f : s.r.inv.z};
  } else {
    R.ird = safe_inverse(rd);
  }
  R.inst = inst;
  return true;
}

// the first instance from `inst` on whose grid the ray overlaps; false when
// none is left
__device__ __forceinline__ bool shadow_ray_next(const DevAccel &A, ShadowRay &R, DdaState &s, uint32_t inst, f3 o,
                                                f3 d) {
  for (; inst < A.n_grids; inst++)
    if (shadow_ray_instance(A, R, s, inst, o, d)) return true;
  return false;
}

// is_vertex_visible's set-up (light.glsl:82-105): the target voxel's key by
// its own box test, then the first instance to walk.  False: nothing to walk
// (the ray is visible).
__device__ __forceinline__ bool shadow_ray_begin(const DevAccel &A, ShadowRay &R, DdaState &s, f3 o, f3 d,
                                                 float distance, uint32_t t_inst, uint32_t t_prim,
                                                 bool check_instance) {
  R.tmax = distance;
  R.target_t = INFINITY;
  R.target_g = 0xFFFFFFFFu;
  const bool has_target = check_instance && t_inst < A.n_grids;
  R.target_inst = has_target ? t_inst : 0xFFFFFFFFu;
  R.target_prim = t_prim;
  if (has_target) {
    const DevGrid &g = A.grids[t_inst];
    if (t_prim < g.primitive_count) {
      const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
      const uint32_t gp = g.first_primitive_index + t_prim;
      const uint32_t pk = __ldg(&A.voxel_coord[gp]);
      const int x = (int)(pk & 0x3FFu), y = (int)((pk >> 10) & 0x3FFu), z = (int)((pk >> 20) & 0x3FFu);
      const f3 ro = xyz(mul(g.world2obj_inst, mk4(o, 1.0f)));
      const f3 rd = xyz(mul(g.world2obj_inst, mk4(d, 0.0f)));
      const f3 ird = safe_inverse(rd);
      const BoxHit h = box_test(voxel_center(A, g, x, y, z, t_prim), radius, inv_radius, ro, rd, false, false, ird);
      if (h.hit && h.t >= 0.f && h.t <= distance) { R.target_t = h.t; R.target_g = gp; }
      // the first instance to walk is usually the target's: its
      // object-space ray is the one just made
      if (t_inst == 0u) {
        if (shadow_ray_instance(A, R, s, 0u, o, d, true, ro, rd, ird)) return true;
        return shadow_ray_next(A, R, s, 1u, o, d);
      }
    }
  }
  return shadow_ray_next(A, R, s, 0, o, d);
}

// QueryVisitor::visit in visibility mode on the stored ray: true when voxel
// (x, y, z) = primitive `prim` of the instance blocks the ray
__device__ __forceinline__ bool shadow_blocks(const DevAccel &A, const DevGrid &g, const ShadowRay &R, int x, int y,
                                              int z, uint32_t prim) {
  if (R.inst == R.target_inst && prim == R.target_prim) return false;
  const f3 radius = half_extent_v(A), inv_radius = safe_inverse(radius);
  const BoxHit h = box_test(voxel_center(A, g, x, y, z, prim), radius, inv_radius, R.ro, R.rd, false, false, R.ird);
  if (!h.hit) return false;
  const float t = h.t;
  if (!(t >= 0.f && t <= R.tmax)) return false;
  const uint32_t gp = g.first_primitive_index + prim;
  return t < R.target_t || (t == R.target_t && gp < R.target_g);
}

// A dilated cell's job: cell (cx, cy, cz) crossed over [t_in, t_out],
// entered across `entry` (-1: the walk began in it) and left across `exit`.
// Packed: x = cx | cy << 16, y = cz | lane << 16 | (entry + 1) << 24 | exit << 28.
__device__ __forceinline__ uint4 shadow_job(int cx, int cy, int cz, float t_in, float t_out, int entry, int exit,
                                            uint32_t lane) {
  return make_uint4((uint32_t)cx | ((uint32_t)cy << 16),
                    (uint32_t)cz | (lane << 16) | ((uint32_t)(entry + 1) << 24) | ((uint32_t)exit << 28),
                    __float_as_uint(t_in), __float_as_uint(t_out));
}
__device__ __forceinline__ uint32_t shadow_job_lane(uint4 j) { return (j.y >> 16) & 31u; }

// The tests of one job, those dda_run makes in a dilated cell: the cell's own
// voxel, then the neighbours the ray passes within eps of.
__device__ __forceinline__ bool shadow_job_blocked(const DevAccel &A, const ShadowRay &R, uint4 j, uint32_t &tests) {
  const DevGrid &g = A.grids[R.inst];
  const int cx = (int)(j.x & 0xFFFFu), cy = (int)(j.x >> 16), cz = (int)(j.y & 0xFFFFu);
  const int entry = (int)((j.y >> 24) & 15u) - 1, ax = (int)(j.y >> 28);
  const float t_in = __uint_as_float(j.z), t_out = __uint_as_float(j.w);
  const int32_t own = voxel_prim(A, g, cx, cy, cz);
  if (own >= 0) {
    tests++;
    if (shadow_blocks(A, g, R, cx, cy, cz, (uint32_t)own)) return true;
  }
  const int sx = ct_step_of(R.r.d.x), sy = ct_step_of(R.r.d.y), sz = ct_step_of(R.r.d.z);
  const int c3[3] = {cx, cy, cz}, st3[3] = {sx, sy, sz};
  if (!dda_near_faces(R.r, c3, t_in, t_out, entry, ax, st3)) return false;
  for (uint32_t m = dda_neighbour_mask(R.r, cx, cy, cz, t_in, t_out, entry, ax, sx, sy, sz); m; m &= m - 1u) {
    const int k = __ffs(m) - 1;
    const int x = cx + k % 3 - 1, y = cy + (k / 3) % 3 - 1, z = cz + k / 9 - 1;
    const int32_t pr = voxel_prim(A, g, x, y, z);
    if (pr < 0) continue;
    tests++;
    if (shadow_blocks(A, g, R, x, y, z, (uint32_t)pr)) return true;
  }
  return false;
}

// One step of dda_run without its visits: leaves the current box; a single
// cell with a test to make sets `job` (its tests are the caller's).  `stop`
// is the visitor's fixed stop distance.  DDA_MORE, DDA_DONE (left the grid or
// passed the stop distance) or DDA_LIMIT.  A step makes one dependent load,
// the cell field's word, and spends the rest of its issue slots on box
// arithmetic and the side-face screen.
__device__ __forceinline__ int shadow_step(const DevAccel &A, const DevGrid &g, const DdaRay &r, DdaState &s, float stop,
                                           uint32_t lane, RayStats &rs, bool &job, uint4 &jb) {
  job = false;
  if (++s.steps > CT_DDA_MAX_STEPS) return DDA_LIMIT;
  const int sx = ct_step_of(r.d.x), sy = ct_step_of(r.d.y), sz = ct_step_of(r.d.z);
  const int cx = s.cx, cy = s.cy, cz = s.cz;
  const int bkey = (cx >> 3) | ((cy >> 3) << 10) | ((cz >> 3) << 20);  // bricks per axis < 1024
  if (bkey != s.cur_bkey) {
    rs.bricks++;
    s.cur_bkey = bkey;
  }
  const int k = cell_field(A, g, ct_ray_octant(sx, sy, sz), cx, cy, cz);
  const int gx = g.bdim[0] * CT_BRICK, gy = g.bdim[1] * CT_BRICK, gz = g.bdim[2] * CT_BRICK;
  int lox, hix, loy, hiy, loz, hiz;
  ct_box_axis(cx, sx, k, gx, lox, hix);
  ct_box_axis(cy, sy, k, gy, loy, hiy);
  ct_box_axis(cz, sz, k, gz, loz, hiz);
  float tb = INFINITY;
  int ax = 0;
  ct_box_exit(0, sx, lox, hix, r.o.x, r.inv.x, tb, ax);
  ct_box_exit(1, sy, loy, hiy, r.o.y, r.inv.y, tb, ax);
  ct_box_exit(2, sz, loz, hiz, r.o.z, r.inv.z, tb, ax);
  if (ct_screen_box(r, k, cx, cy, cz, sx, sy, sz, s.t_in, s.entry_axis, lox, hix, loy, hiy, loz, hiz, tb, ax)) {
    // a job only when it has a test to make: the cell's own voxel, or a
    // neighbour face the ray passes near
    const int c3[3] = {cx, cy, cz}, st3[3] = {sx, sy, sz};
    if (k == 0 || dda_near_faces(r, c3, s.t_in, tb, s.entry_axis, ax, st3)) {
      job = true;
      jb = shadow_job(cx, cy, cz, s.t_in, tb, s.entry_axis, ax, lane);
    }
  }
  // dda_run's end test (see there for the slack)
  const float slack = ((r.eps - 2e-4f) * 0.25f + 1e-6f) * fabsf(ax == 0 ? r.inv.x : (ax == 1 ? r.inv.y : r.inv.z));
  if (tb - slack > stop + 1e-5f * fabsf(stop) + 1e-6f || tb - slack >= s.t1) return DDA_DONE;
  const int nx = ct_box_next(ax == 0, sx, lox, hix, r.d.x, tb, r.o.x);
  const int ny = ct_box_next(ax == 1, sy, loy, hiy, r.d.y, tb, r.o.y);
  const int nz = ct_box_next(ax == 2, sz, loz, hiz, r.d.z, tb, r.o.z);
  const bool out = ax == 0 ? (nx < 0 || nx >= gx) : (ax == 1 ? (ny < 0 || ny >= gy) : (nz < 0 || nz >= gz));
  if (out) return DDA_DONE;
  s.cx = nx; s.cy = ny; s.cz = nz;
  s.t_in = tb;
  s.entry_axis = ax;
  return DDA_MORE;
}

// ---------------------------------------------------------------------------
// Unit axis vectors (one component +-1, the others +-0) are what voxel faces
// give for normals.  normalize() returns them unchanged, bit for bit (the
// length is exactly 1 and x/1 == x, signed zeros included), so the helpers
// below skip the square root and the divisions for them.
__device__ __forceinline__ bool is_unit_axis(f3 v) {
  const float ax = fabsf(v.x), ay = fabsf(v.y), az = fabsf(v.z);
  return (ax == 1.0f && ay == 0.0f && az == 0.0f) || (ax == 0.0f && ay == 1.0f && az == 0.0f) ||
         (ax == 0.0f && ay == 0.0f && az == 1.0f);
}
__device__ __forceinline__ f3 normalize_n(f3 v) { return is_unit_axis(v) ? v : normalize(v); }

// materials (mat.glsl:24-88, light.glsl:200-229)
__device__ __forceinline__ void orthonormal_basis(f3 n, f3 &t1, f3 &t2) {
  if (fabsf(n.x) > fabsf(n.y)) t1 = normalize_n(f3{-n.z, 0.0f, n.x});
  else t1 = normalize_n(f3{0.0f, n.z, -n.y});
  t2 = normalize_n(cross(n, t1));
}
// z component of to_local(n, v) = dot(v, normalize(n)) (mat.glsl:58-64); the
// other two components are dot(u,w) and dot(v2,w) of the basis and unused by
// the Lambertian lobe.
__device__ __forceinline__ float local_z(f3 n, f3 v) { return dot(v, normalize_n(n)); }

__device__ __forceinline__ f3 evaluate_material(const Material &m, f3 n, f3 wo, f3 wi) {
  switch (m.type & 0xFFu) {
    case 1u: {  // metal (mat.glsl:30-36)
      f3 half_dir = normalize(wi + wo);
      float r = gmin(m.roughness, 1.0f);
      float p = ct_powf(1.0f - dot(wi, half_dir), 5.0f);
      f3 fres = mk3(r) + (mk3(1.0f) - mk3(r)) * p;
      f3 diff = (mk3(1.0f) - fres) * (mk3(1.0f) - m.specular);
      f3 spec = fres * m.specular;
      return (diff + spec) * 0.31830988618379067153776752674503f;
    }
    case 2u: {  // dielectric (mat.glsl:38-50)
      float p = ct_powf(1.0f - dot(wi, wo), 5.0f);
      f3 fres = mk3(m.roughness) + (mk3(1.0f) - mk3(m.roughness)) * p;
      f3 diff = (mk3(1.0f) - fres) * (m.diffuse * 0.31830988618379067153776752674503f);
      return diff + fres;
    }
    case 3u:  // constant medium (mat.glsl:53-55)
      return m.diffuse * 0.079577471545947667884441881686255f;
    default: {
      float wo_z = local_z(n, wo), wi_z = local_z(n, wi);
      if (gmin(wo_z, wi_z) < 1e-6f) return mk3(0.f);
      return m.diffuse * 0.31830988618379067153776752674503f * wi_z;
    }
  }
}
__device__ __forceinline__ float sample_material_pdf(const Material &m, f3 n, f3 wo, f3 wi) {
  switch (m.type & 0xFFu) {
    case 1u: case 2u: return 6.283185307179586476925286766559f;
    case 3u: return 12.566370614359172953850573533118f;
    default: {
      float wo_z = local_z(n, wo), wi_z = local_z(n, wi);
      if (gmin(wo_z, wi_z) < 1e-6f) return 0.f;
      return 0.31830988618379067153776752674503f * wi_z;
    }
  }
}

// ---------------------------------------------------------------------------
// light sampling (light.glsl:160-164, 295-435; prng.glsl:64-173)
__device__ __forceinline__ float geom_fact_sa(f3 P, f3 Ps, f3 ns) {
  f3 dir = normalize(Ps - P);
  float dist2 = dot(Ps - P, Ps - P);
  return fabsf(dot(ns, dir)) / dist2;
}
__device__ __forceinline__ f3 random_cube_normal(uint32_t &seed) {
  uint32_t face = gmin(urnd_interval(seed, 0u, 6u), 5u);
  switch (face) {
    case 0: return f3{-1.f, 0.f, 0.f};
    case 1: return f3{1.f, 0.f, 0.f};
    case 2: return f3{0.f, -1.f, 0.f};
    case 3: return f3{0.f, 1.f, 0.f};
    case 4: return f3{0.f, 0.f, -1.f};
    default: return f3{0.f, 0.f, 1.f};
  }
}
__device__ __forceinline__ f3 random_quad(f3 n, f3 p, f2 s, uint32_t &seed) {
  float u = rnd(seed);
  float v = rnd(seed);
  f2 q = f2{u, v} * s;
  f3 xa, ya;
  orthonormal_basis(n, xa, ya);
  return p + xa * q.x + ya * q.y;
}
__device__ __forceinline__ f3 random_unit_vector(uint32_t &seed, uint32_t pixel) {
  f3 p = f3{0.f, 0.f, 0.f};
  for (int i = 0; i < CT_SAMPLER_MAX_TRIES; i++) {
    float a = -1.0f + rnd(seed) * (1.0f - -1.0f);
    float b = -1.0f + rnd(seed) * (1.0f - -1.0f);
    float c = -1.0f + rnd(seed) * (1.0f - -1.0f);
    p = f3{a, b, c};
    if (p.x * p.x + p.y * p.y + p.z * p.z >= 1.0f) {
      if (i == CT_SAMPLER_MAX_TRIES - 1) ct_latch_error(CT_ERR_ITER_LIMIT, 3, pixel);
      continue;
    }
    break;
  }
  return normalize(p);
}

struct LightSample {
  bool vis;
  f3 l_pos, l_nor, Le;
  float G;
  bool g_set;
};

// sample_lights: chooses a point on `l` as seen from the shading point, its
// pdf update, and (when `visibility`) asks the visibility provider `vp` about
// the shadow ray; `slot` names the call site so that a later pass can find
// the answer (see VisEmit / VisRead).
template <class VP>
__device__ LightSample sample_lights(const FrameView &F, f3 P, f3 n, uint32_t hit_inst, uint32_t hit_prim, Light l,
                                     float &pdf, uint32_t &seed, bool calc_pdf, bool visibility, uint32_t pixel,
                                     VP &vp, uint32_t slot) {
  LightSample s;
  s.g_set = false;
  s.G = 0.f;
  s.l_pos = mk3(0.f);
  s.l_nor = mk3(0.f);
  if (l.inst == hit_inst && l.prim == hit_prim) { s.vis = false; s.Le = mk3(0.f); return s; }
  bool vis = true, check_instance = false;
  float distance = -1.0f;
  f3 l_wi = mk3(0.f), l_pos = mk3(0.f), l_nor = mk3(0.f);
  if (l.type == CT_LIGHT_CUBE) {
    float half_extent = l.size * 0.5f;
    f2 quad = f2{l.size, l.size};
    uint32_t i = 0;
    // With l_nor and n unit axis vectors, dot(normalize(v), axis) is the
    // one product v_k / |v| * (+-1) plus signed zeros, whose sign is that of
    // v_k * (+-1): the tries test signs and normalise only the last vector.
    const bool fast = is_unit_axis(n);
    // A try succeeds only for a point in front of the shading point's plane
    // (dot(P - l_pos, n) < 0).  When the whole cube lies behind that plane,
    // by a margin far above the rounding of l_pos, all 11 tries fail and the
    // first 10 only advance the RNG (3 draws each: a face, two quad
    // coordinates): jump over their 30 draws and run the last try, which
    // leaves l_pos, l_nor and the seed exactly as the full loop does.
    {
      const f3 c = l.position - P;
      const float reach = dot(c, n) + half_extent * (fabsf(n.x) + fabsf(n.y) + fabsf(n.z));
      const float scale = fmaxf(fmaxf(fmaxf(fabsf(P.x), fabsf(P.y)), fmaxf(fabsf(P.z), fabsf(l.position.x))),
                                fmaxf(fmaxf(fabsf(l.position.y), fabsf(l.position.z)), l.size));
      if (reach < -1e-5f * scale) {
        seed = lcg_jump<30>(seed);
        i = 10;
      }
    }
    do {
      vis = true;
      l_nor = random_cube_normal(seed);
      l_pos = l.position + l_nor * half_extent;
      l_pos = random_quad(l_nor, l_pos, quad * 0.5f, seed);
      if (fast) {
        const f3 v = P - l_pos;
        vis = vis && (v.x * l_nor.x + v.y * l_nor.y + v.z * l_nor.z > 0.0f);
        vis = vis && (v.x * n.x + v.y * n.y + v.z * n.z < 0.0f);
      } else {
        l_wi = normalize(P - l_pos);
        vis = vis && (dot(l_wi, l_nor) > 0.0f);
        vis = vis && (dot(l_wi, n) < 0.0f);
      }
    } while (!vis && i++ < 10);
    if (fast) l_wi = normalize(P - l_pos);
    l_pos = offset_twice(l_pos, l_nor);
    distance = length(P - l_pos);
    if (calc_pdf) {
      float area = quad.x * quad.y * 6.0f;
      pdf = pdf / area;
    }
    check_instance = true;
    s.G = geom_fact_sa(P, l_pos, l_nor);
    s.g_set = true;
  } else if (l.type == CT_LIGHT_POINT) {
    l_pos = l.position;
    l_nor = normalize(P - l_pos);
    distance = length(P - l_pos);
    l_wi = l_nor;
    s.G = geom_fact_sa(P, l_pos, l_nor);
    s.g_set = true;
  } else if (l.type == CT_LIGHT_ENV_MAP) {
    f3 u = random_unit_vector(seed, pixel);
    f3 l_dir = dot(u, n) > 0.0f ? u : -u;
    l_pos = P + (l_dir * 1e9f);
    l_nor = normalize(P - l_pos);
    distance = length(P - l_pos);
    l_wi = l_nor;
    l.emissive = l.emissive * sky_color(F.time, F.is_afternoon, l_dir);
    if (calc_pdf) pdf = pdf / 0.079577471545947667884441881686255f;
    s.G = 1.0f;
    s.g_set = true;
  }
  f3 l_v = -l_wi;
  if (visibility && vis) vis = vis && vp(P, l_v, distance, l.inst, l.prim, check_instance, slot);
  s.vis = vis;
  s.l_pos = l_pos;
  s.l_nor = l_nor;
  s.Le = vis ? l.emissive : mk3(0.f);
  return s;
}

// calculate_sampled_light (light.glsl:401-435).  `scatter_dir` is the
// HIT_INFO_INPUT.scatter_dir the shader updates in place; `G` stays 0 when the
// sampler returns before computing it (the shader leaves it unset).
template <class VP>
__device__ f3 calculate_sampled_light(const FrameView &F, f3 ray_dir, f3 P, f3 n, uint32_t hit_inst, uint32_t hit_prim,
                                      const Material &mat, const Light &light, float pdf, float &pdf_out, float &G,
                                      uint32_t &seed, bool calc_pdf, bool use_pdf, bool use_visibility,
                                      f3 &scatter_dir, uint32_t pixel, VP &vp, uint32_t slot) {
  f3 surface_normal = normalize_n(n);
  f3 wo = -normalize(ray_dir);
  pdf_out = pdf;
  G = 0.f;
  f3 result = mk3(0.f);
  if (all_le_zero(light.emissive)) return result;
  LightSample s = sample_lights(F, P, n, hit_inst, hit_prim, light, pdf_out, seed, calc_pdf, use_visibility, pixel, vp,
                                slot);
  if (s.g_set) G = s.G;
  if (s.vis) {
    f3 wi = normalize(s.l_pos - P);
    f3 brdf = evaluate_material(mat, surface_normal, wo, wi);
    scatter_dir = wi;
    if (use_pdf) result = brdf * s.Le * G / pdf_out;
    else result = brdf * s.Le * G;
  }
  return result;
}

// ---------------------------------------------------------------------------
// reservoirs (reservoir.glsl:17-126)
struct Reservoir {
  uint32_t Y, l_type, seed;
  float W_y, W_sum, M;
  f3 F;
};
__device__ __forceinline__ Reservoir reservoir_empty() {
  Reservoir r;
  r.W_y = 0.f; r.seed = 0; r.W_sum = 0.f; r.M = 0.f; r.Y = 0xFFFFFFFFu; r.l_type = CT_LIGHT_NONE; r.F = mk3(0.f);
  return r;
}
__device__ __forceinline__ Reservoir load_reservoir(const ct_reservoir *b, uint32_t i) {
  const ct_reservoir &s = b[i];
  Reservoir r;
  r.Y = s.Y; r.l_type = s.l_type; r.seed = s.seed; r.W_y = s.W_y; r.W_sum = s.W_sum; r.M = s.M; r.F = ld3(s.F);
  return r;
}
__device__ __forceinline__ void store_reservoir(ct_reservoir *b, uint32_t i, const Reservoir &r) {
  ct_reservoir &s = b[i];
  s.Y = r.Y; s.l_type = r.l_type; s.seed = r.seed; s.W_y = r.W_y; s.W_sum = r.W_sum; s.M = r.M; st3(s.F, r.F);
}
__device__ __forceinline__ bool update_reservoir(Reservoir &r, uint32_t X, uint32_t l_type, uint32_t random_seed, f3 Fv,
                                                 float w, float c, uint32_t &seed) {
  if (w < 0.0f || isnan(w) || isinf(w)) return false;
  r.M += c;
  r.W_sum += w;
  if (rnd(seed) < (w / r.W_sum)) {
    r.Y = X; r.l_type = l_type; r.seed = random_seed; r.F = Fv;
    return true;
  }
  return false;
}
__device__ __forceinline__ bool reservoir_valid(const Reservoir &r) {
  return r.M > 0.0f && r.Y != 0xFFFFFFFFu && r.l_type != CT_LIGHT_NONE;
}

// shading point of a DI info record, as every pass reconstructs it
struct Shade {
  f3 P;          // compute_ray_origin(position, normal) applied twice
  f3 n;
  float distance;
  uint32_t inst, prim, mat_index;
};

// reservoir_get_radiance (reservoir.glsl:98-112): re-evaluates the reservoir's
// sample, replaying its stored light seed, with a shadow ray.
template <class VP>
__device__ f3 reservoir_get_radiance(const FrameView &F, const Reservoir &r, f3 ray_dir, const Shade &s,
                                     const Material &mat, uint32_t pixel, VP &vp, uint32_t slot) {
  if (!reservoir_valid(r)) return mk3(0.f);
  Light light = light_get_by_type(F, r.l_type, r.Y);
  uint32_t seed = r.seed;
  float pdf_out, G;
  f3 scatter = mk3(0.f);
  return calculate_sampled_light(F, ray_dir, s.P, s.n, s.inst, s.prim, mat, light, 1.0f, pdf_out, G, seed, false,
                                 false, true, scatter, pixel, vp, slot);
}

// ---------------------------------------------------------------------------
// Visibility providers.  The shading passes run twice over a pixel: the
// generating pass records every shadow ray the shader would trace (VisEmit,
// into a compacted queue traced by k_trace_shadow), the resolving pass
// replays the same deterministic light samples and reads the answers back
// (VisRead).  A call site traces at most one ray and owns one fixed slot.
#define CT_VIS_SLOTS 16u  // per pixel: 2 per spatial neighbour; stage 0 uses 0..2

struct RayQueue {
  float4 *a;        // origin.xyz, distance
  float4 *b;        // direction.xyz, result slot (bits)
  uint2 *c;         // target (instance | check flag << 31, primitive)
  uint32_t *count;
  uint32_t capacity;
};

struct VisNever {  // for samplers called with visibility off
  __device__ bool operator()(f3, f3, float, uint32_t, uint32_t, bool, uint32_t) { return true; }
};

// Generating passes run their shadow-ray call sites twice: VisCount counts
// the rays a thread will emit, block_reserve (a block-wide scan, one atomic
// per block) turns the counts into queue positions, and VisEmit writes the
// rays there.  Every thread of the block must reach block_reserve.
struct VisCount {
  uint32_t n;
  __device__ bool operator()(f3, f3, float, uint32_t, uint32_t, bool, uint32_t) { n++; return true; }
};

struct VisEmit {
  RayQueue q;
  uint32_t base;  // pixel * CT_VIS_SLOTS
  uint32_t pixel;
  uint32_t next;  // queue position of this thread's next ray
  __device__ bool operator()(f3 o, f3 d, float dist, uint32_t inst, uint32_t prim, bool check, uint32_t slot) {
    const uint32_t i = next++;
    if (i >= q.capacity) { ct_latch_error(CT_ERR_CAPACITY, 5, pixel); return true; }
    q.a[i] = make_float4(o.x, o.y, o.z, dist);
    q.b[i] = make_float4(d.x, d.y, d.z, __uint_as_float(base + slot));
    q.c[i] = make_uint2(inst | (check ? 0x80000000u : 0u), prim);
    return true;
  }
};

// Exclusive prefix of `n` over the block plus one atomicAdd on `counter`;
// returns this thread's first position.  Blocks are whole warps.
__device__ __forceinline__ uint32_t block_reserve(uint32_t n, uint32_t *counter) {
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t block_base;
  const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x;
  const uint32_t lane = tid & 31u, wid = tid >> 5;
  const uint32_t nwarps = (blockDim.x * blockDim.y + 31u) >> 5;
  uint32_t incl = n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (uint32_t)o) incl += v;
  }
  if (lane == 31u) warp_sum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = lane < nwarps ? warp_sum[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= (uint32_t)o) wi += v;
    }
    if (lane < nwarps) warp_sum[lane] = wi - w;
    if (lane == nwarps - 1u) block_base = wi ? atomicAdd(counter, wi) : 0u;
  }
  __syncthreads();
  return block_base + warp_sum[wid] + incl - n;
}

struct VisRead {
  const uint8_t *vis;
  uint32_t base;
  __device__ bool operator()(f3, f3, float, uint32_t, uint32_t, bool, uint32_t slot) { return vis[base + slot] != 0; }
};

__device__ __forceinline__ Shade shade_from_di(const ct_di_info &d) {
  Shade s;
  f3 pos = ld3(d.position);
  s.n = ld3(d.normal);
  s.P = offset_twice(pos, s.n);
  s.distance = d.distance;
  s.inst = d.instance_hit.instance_id;
  s.prim = d.instance_hit.primitive_id;
  s.mat_index = d.mat_index;
  return s;
}

#define CT_HLF_MAX 6.5504e+4f
#define CT_HLF_MIN 1.175494351e-38f

// The dielectric scatter callable's first step (rcall_scatter.glsl:20-30): a
// normal that faces along the ray is turned and the point pushed through the
// face.  The callable works on the caller's hit record (sample_material,
// light.glsl:231-260, takes it inout).
__device__ __forceinline__ bool dielectric_face(f3 &hit, f3 &nrm, f3 ray_dir) {
  if (!(dot(ray_dir, nrm) > 0.0f)) return false;
  nrm = -nrm;
  hit = hit - nrm * CT_HLF_MIN * 2.0f;
  return true;
}

// The shading point the rest of the first pass sees after RIS.  The BRDF
// candidates (restir_resampling.glsl:193-230) hand the pass's hit record to
// sample_material, so on a dielectric hit from behind its face the record
// leaves RIS turned: the RIS visibility pass and TEMPORAL_REUSE that follow
// in the same invocation (rgen.glsl:255-262) work on the turned record, while
// the DI record and everything after the first pass keep the hit as found.
// Only the first candidate can turn it (the turned normal faces the ray).
__device__ __forceinline__ void turn_after_ris(const FrameView &F, Shade &S, f3 ray_dir) {
  if (!(F.is_active & CT_RIS_BRDF_BIT) || F.light_config.brdf_count == 0u) return;
  if ((F.materials[S.mat_index].type & 0xFFu) != 2u) return;
  dielectric_face(S.P, S.n, ray_dir);
}
