// ct_math.cuh -- single-precision vector math with the exact operation order
// the hot path's results depend on.
//
// The ray-tracing shaders this library replaces are GLSL; GLSL leaves the
// precise sequence of some operations to the implementation.  To make results
// reproducible (and comparable bit for bit with a CPU build of the same
// shaders) every helper here fixes one order, and the library is compiled
// with --fmad=false so that no multiply-add is contracted behind our back:
//
//   dot(a,b)     = (a.x*b.x + a.y*b.y) + a.z*b.z
//   normalize(v) = v / sqrt(dot(v,v)), one IEEE division per component
//   mix(x,y,a)   = x*(1-a) + y*a
//   min(x,y)     = y < x ? y : x,   max(x,y) = x < y ? y : x   (GLSL 4.60 8.3)
//   M*v          = ((c0*v.x + c1*v.y) + c2*v.z) + c3*v.w
//   inverse(M)   = cofactor expansion / determinant (ct_inverse below)
//   float->uint  = truncating, saturating, NaN -> 0 (cvt.rzi.u32.f32)
//
// Code that does not feed a parity-checked result (the DDA stepping in the
// traversal) is free to use fused operations explicitly.
#pragma once
#include <cstdint>
#include <cstring>

#define CT_HD __host__ __device__ __forceinline__

struct f2 { float x, y; };
struct f3 { float x, y, z; };
struct f4 { float x, y, z, w; };
struct m4 { f4 c[4]; };  // column major

CT_HD f2 mk2(float x, float y) { return f2{x, y}; }
CT_HD f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
CT_HD f3 mk3(float s) { return f3{s, s, s}; }
CT_HD f4 mk4(float x, float y, float z, float w) { return f4{x, y, z, w}; }
CT_HD f4 mk4(f3 v, float w) { return f4{v.x, v.y, v.z, w}; }
CT_HD f3 xyz(f4 v) { return f3{v.x, v.y, v.z}; }

CT_HD f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
CT_HD f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
CT_HD f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
CT_HD f3 operator/(f3 a, f3 b) { return f3{a.x / b.x, a.y / b.y, a.z / b.z}; }
CT_HD f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
CT_HD f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
CT_HD f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
CT_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
CT_HD f3 operator+(f3 a, float s) { return f3{a.x + s, a.y + s, a.z + s}; }
CT_HD f2 operator+(f2 a, f2 b) { return f2{a.x + b.x, a.y + b.y}; }
CT_HD f2 operator-(f2 a, f2 b) { return f2{a.x - b.x, a.y - b.y}; }
CT_HD f2 operator*(f2 a, f2 b) { return f2{a.x * b.x, a.y * b.y}; }
CT_HD f2 operator/(f2 a, f2 b) { return f2{a.x / b.x, a.y / b.y}; }
CT_HD f2 operator*(f2 a, float s) { return f2{a.x * s, a.y * s}; }
CT_HD f2 operator*(float s, f2 a) { return f2{s * a.x, s * a.y}; }
CT_HD f2 operator/(f2 a, float s) { return f2{a.x / s, a.y / s}; }
CT_HD f2 operator-(f2 a, float s) { return f2{a.x - s, a.y - s}; }
CT_HD f2 operator+(f2 a, float s) { return f2{a.x + s, a.y + s}; }
CT_HD f4 operator+(f4 a, f4 b) { return f4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
CT_HD f4 operator*(f4 a, float s) { return f4{a.x * s, a.y * s, a.z * s, a.w * s}; }
CT_HD f4 operator*(float s, f4 a) { return f4{s * a.x, s * a.y, s * a.z, s * a.w}; }
CT_HD f4 operator/(f4 a, float s) { return f4{a.x / s, a.y / s, a.z / s, a.w / s}; }

CT_HD float gmin(float x, float y) { return y < x ? y : x; }
CT_HD float gmax(float x, float y) { return x < y ? y : x; }
CT_HD uint32_t gmin(uint32_t x, uint32_t y) { return y < x ? y : x; }
CT_HD uint32_t gmax(uint32_t x, uint32_t y) { return x < y ? y : x; }
CT_HD float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
CT_HD float gmix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
CT_HD f3 gmix(f3 x, f3 y, float a) { return x * (1.0f - a) + y * a; }
CT_HD float gsign(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
CT_HD f3 gsign(f3 v) { return f3{gsign(v.x), gsign(v.y), gsign(v.z)}; }
CT_HD f3 gabs(f3 v) { return f3{fabsf(v.x), fabsf(v.y), fabsf(v.z)}; }
CT_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CT_HD float dot(f4 a, f4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
CT_HD float length(f3 v) { return sqrtf(dot(v, v)); }
CT_HD f3 normalize(f3 v) { float l = length(v); return f3{v.x / l, v.y / l, v.z / l}; }
CT_HD f3 cross(f3 a, f3 b) { return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
CT_HD bool any_nan_inf(f3 v) { return isnan(v.x) || isnan(v.y) || isnan(v.z) || isinf(v.x) || isinf(v.y) || isinf(v.z); }
CT_HD bool all_le_zero(f3 v) { return v.x <= 0.f && v.y <= 0.f && v.z <= 0.f; }

// luminance (light.glsl:78-80)
CT_HD float luminance(f3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

CT_HD f4 mul(const m4 &m, f4 v) {
  return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w;
}
CT_HD m4 mul(const m4 &a, const m4 &b) {
  m4 r;
  for (int i = 0; i < 4; i++) r.c[i] = mul(a, b.c[i]);
  return r;
}
CT_HD m4 load_m4(const float *p) {
  m4 r;
  for (int i = 0; i < 4; i++) r.c[i] = f4{p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]};
  return r;
}
CT_HD float m4_at(const m4 &m, int col, int row) {
  const f4 &c = m.c[col];
  return row == 0 ? c.x : (row == 1 ? c.y : (row == 2 ? c.z : c.w));
}

// 4x4 inverse by cofactor expansion; m[4*col + row].
CT_HD m4 ct_inverse(const m4 &M) {
  float m[16];
  for (int i = 0; i < 4; i++) { m[4 * i] = M.c[i].x; m[4 * i + 1] = M.c[i].y; m[4 * i + 2] = M.c[i].z; m[4 * i + 3] = M.c[i].w; }
  float inv[16];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  float det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  m4 R;
  for (int i = 0; i < 4; i++) R.c[i] = f4{inv[4 * i] / det, inv[4 * i + 1] / det, inv[4 * i + 2] / det, inv[4 * i + 3] / det};
  return R;
}

CT_HD m4 transpose(const m4 &m) {
  m4 r;
  for (int i = 0; i < 4; i++) r.c[i] = f4{m4_at(m, 0, i), m4_at(m, 1, i), m4_at(m, 2, i), m4_at(m, 3, i)};
  return r;
}

// GLSL conversions
#ifdef __CUDA_ARCH__
__device__ __forceinline__ uint32_t f2u(float f) { return __float2uint_rz(f); }
__device__ __forceinline__ int32_t f2i(float f) { return __float2int_rz(f); }
__device__ __forceinline__ int32_t fbits(float f) { return __float_as_int(f); }
__device__ __forceinline__ float bitsf(int32_t i) { return __int_as_float(i); }
#else
inline uint32_t f2u(float f) { if (!(f > 0.f)) return 0u; if (f >= 4294967296.f) return 0xFFFFFFFFu; return (uint32_t)f; }
inline int32_t f2i(float f) { if (f != f) return 0; if (f >= 2147483648.f) return 0x7FFFFFFF; if (f <= -2147483648.f) return (int32_t)0x80000000; return (int32_t)f; }
inline int32_t fbits(float f) { int32_t i; memcpy(&i, &f, 4); return i; }
inline float bitsf(int32_t i) { float f; memcpy(&f, &i, 4); return f; }
#endif

// ---------------------------------------------------------------------------
// random numbers (random.glsl:26-77, prng.glsl): TEA seed hash + the
// Numerical Recipes LCG, 24-bit mantissa floats.
CT_HD uint32_t tea(uint32_t val0, uint32_t val1) {
  uint32_t v0 = val0, v1 = val1, s0 = 0;
#pragma unroll
  for (int n = 0; n < 16; n++) {
    s0 += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return v0;
}
CT_HD uint32_t lcg(uint32_t &prev) {
  prev = 1664525u * prev + 1013904223u;
  return prev & 0x00FFFFFFu;
}
CT_HD float rnd(uint32_t &prev) { return (float)lcg(prev) / (float)0x01000000; }
// K steps of lcg at once: x -> A_K x + C_K (mod 2^32), the constants folded
// at compile time
template <int K>
CT_HD uint32_t lcg_jump(uint32_t x) {
  constexpr uint32_t a = [] {
    uint32_t v = 1u;
    for (int i = 0; i < K; i++) v = 1664525u * v;
    return v;
  }();
  constexpr uint32_t c = [] {
    uint32_t v = 0u;
    for (int i = 0; i < K; i++) v = 1664525u * v + 1013904223u;
    return v;
  }();
  return a * x + c;
}
CT_HD float rnd_interval(uint32_t &prev, float mn, float mx) { return mn + rnd(prev) * (mx - mn); }
CT_HD uint32_t urnd_interval(uint32_t &prev, uint32_t mn, uint32_t mx) {
  if (mn == mx) return mn;
  if (mn > mx) return f2u(rnd_interval(prev, (float)mx, (float)mn));
  return f2u(rnd_interval(prev, (float)mn, (float)mx));
}

// Wachter-Binder self-intersection offset (primitives.glsl:233-257)
CT_HD f3 compute_ray_origin(f3 pos, f3 normal) {
  const float origin = 1.f / 32.f;
  const float f_scale = 1.f / 65536.f;
  const float i_scale = 256.f;
  f3 s = normal * i_scale;
  int32_t ix = f2i(s.x), iy = f2i(s.y), iz = f2i(s.z);
  f3 i_pos;
  i_pos.x = bitsf(fbits(pos.x) + (pos.x < 0.f ? -ix : ix));
  i_pos.y = bitsf(fbits(pos.y) + (pos.y < 0.f ? -iy : iy));
  i_pos.z = bitsf(fbits(pos.z) + (pos.z < 0.f ? -iz : iz));
  f3 f_off = normal * f_scale;
  f3 r;
  r.x = fabsf(pos.x) < origin ? pos.x + f_off.x : i_pos.x;
  r.y = fabsf(pos.y) < origin ? pos.y + f_off.y : i_pos.y;
  r.z = fabsf(pos.z) < origin ? pos.z + f_off.z : i_pos.z;
  return r;
}
CT_HD f3 offset_twice(f3 pos, f3 n) { return compute_ray_origin(compute_ray_origin(pos, n), n); }

CT_HD float safe_inverse(float x) { return (x == 0.0f) ? 1e12f : (1.0f / x); }
CT_HD f3 safe_inverse(f3 v) { return f3{safe_inverse(v.x), safe_inverse(v.y), safe_inverse(v.z)}; }

// cube_like_normal (primitives.glsl:499-507)
CT_HD f3 cube_like_normal(f3 n) {
  f3 a = gabs(n);
  float mc = gmax(gmax(a.x, a.y), a.z);
  return (mc == a.x) ? f3{gsign(n.x), 0.f, 0.f} : ((mc == a.y) ? f3{0.f, gsign(n.y), 0.f} : f3{0.f, 0.f, gsign(n.z)});
}

// Ray / axis-aligned box test of J. Majercik et al., "A Ray-Box Intersection
// Algorithm and Efficient Dynamic Voxel Rendering", JCGT 7(3) 2018, in the
// form cube-tracing uses (primitives.glsl:273-355) with an identity box
// rotation.  The identity products are written out so that signed zeros and
// rounding come out as in the shader.  `o` is the ray origin relative to the
// world, `center` the box centre, `radius` the half extent.
struct BoxHit { bool hit; float t; f3 n; };  // n: intersect_box's normal for oriented = false
CT_HD BoxHit box_test(f3 center, f3 radius, f3 inv_radius, f3 ro, f3 rd, bool can_start_in_box, bool oriented,
                      f3 inv_dir) {
  // ray.origin = rotation * (origin - center), rotation = identity
  f3 v = ro - center;
  f3 o = f3{1.f * v.x + 0.f * v.y + 0.f * v.z, 0.f * v.x + 1.f * v.y + 0.f * v.z, 0.f * v.x + 0.f * v.y + 1.f * v.z};
  f3 d = rd;
  if (oriented)  // direction * rotation (row vector times matrix)
    d = f3{rd.x * 1.f + rd.y * 0.f + rd.z * 0.f, rd.x * 0.f + rd.y * 1.f + rd.z * 0.f, rd.x * 0.f + rd.y * 0.f + rd.z * 1.f};
  float winding = 1.0f;
  if (can_start_in_box) {
    f3 rb = gabs(o) * inv_radius;
    winding = (gmax(rb.x, gmax(rb.y, rb.z)) < 1.0f) ? -1.0f : 1.0f;
  }
  f3 sgn = -gsign(d);
  f3 dp = radius * winding * sgn - o;
  if (oriented) dp = dp / d; else dp = dp * inv_dir;
  bool tx = (dp.x >= 0.0f) && (fabsf(o.y + d.y * dp.x) < radius.y) && (fabsf(o.z + d.z * dp.x) < radius.z);
  bool ty = (dp.y >= 0.0f) && (fabsf(o.z + d.z * dp.y) < radius.z) && (fabsf(o.x + d.x * dp.y) < radius.x);
  bool tz = (dp.z >= 0.0f) && (fabsf(o.x + d.x * dp.z) < radius.x) && (fabsf(o.y + d.y * dp.z) < radius.y);
  f3 s = tx ? f3{sgn.x, 0.f, 0.f} : (ty ? f3{0.f, sgn.y, 0.f} : f3{0.f, 0.f, tz ? sgn.z : 0.f});
  BoxHit r;
  r.t = (s.x != 0.f) ? dp.x : ((s.y != 0.f) ? dp.y : dp.z);
  r.hit = (s.x != 0.f) || (s.y != 0.f) || (s.z != 0.f);
  r.n = s;
  return r;
}
