// glsl_shim.hpp -- GLSL semantics for compiling the cube-tracing shader
// sources (src/shaders/**.glsl) as plain C++ on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  This header is part of the parity oracle: it
// lets the reference's own GLSL for the per-pixel hot path run on host cores
// so that the CUDA kernels can be checked against it.  Nothing in the product
// library links or includes it.
//
// Every arithmetic helper below fixes one evaluation order.  The GLSL spec
// leaves some of these implementation-defined (normalize, mix, inverse, the
// summation order of matrix products); the CUDA kernels use the same
// definitions so both sides round identically.  Build with
// -ffp-contract=off (no FMA contraction) and without -ffast-math.
//
//   dot(a,b)      = ((a.x*b.x) + a.y*b.y) + a.z*b.z              (left to right)
//   length(v)     = sqrt(dot(v,v))
//   normalize(v)  = v / length(v)            (three IEEE divisions)
//   mix(x,y,a)    = x*(1-a) + y*a            (GLSL 4.60 section 8.3 definition)
//   min(x,y)      = y < x ? y : x            (GLSL 4.60 section 8.3 definition)
//   max(x,y)      = x < y ? y : x
//   clamp(x,l,h)  = min(max(x,l),h)
//   M*v           = ((c0*v.x + c1*v.y) + c2*v.z) + c3*v.w   (column major)
//   v*M           = (dot(v,c0), dot(v,c1), dot(v,c2), ...)
//   inverse(M)    = adjugate / determinant, cofactor expansion below
//   float->uint   = saturating, truncating (negative and NaN -> 0), which is
//                   the conversion CUDA's cvt.rzi.u32.f32 performs
//
// Function arguments: GLSL evaluates them left to right.  C++ does not
// guarantee that for calls, so the oracle's source transform rewrites vector
// and struct constructor calls into brace-initialisation, which C++ does
// sequence left to right.
#pragma once
#include "ct_fpmath.h"
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

typedef uint32_t uint;

// The shaders' floating-point type.  The parity oracle is single precision,
// as the shaders are; the FP64 build (CT_ORACLE_FP64) evaluates the same code
// in double precision to state the single-precision results' error, keeping
// compute_ray_origin's FP32 bit arithmetic (floatBitsToInt below).
#ifdef CT_ORACLE_FP64
typedef double ct_real;
#else
typedef float ct_real;
#endif

// ---------------------------------------------------------------------------
// scalar conversions with GLSL semantics
static inline uint32_t glsl_u32_from_f(double f) {
  if (!(f > 0.0)) return 0u;               // negative, zero, NaN
  if (f >= 4294967296.0) return 0xFFFFFFFFu;
  return (uint32_t)f;                      // truncation
}
template <class T> static inline uint32_t glsl_u32(T v) {
  if constexpr (std::is_floating_point<T>::value) return glsl_u32_from_f((double)v);
  else return (uint32_t)v;
}
template <class T> static inline int32_t glsl_i32(T v) {
  if constexpr (std::is_floating_point<T>::value) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483648.0) return 0x7FFFFFFF;
    if (v <= -2147483648.0) return (int32_t)0x80000000;
    return (int32_t)v;
  } else return (int32_t)v;
}
template <class T> static inline ct_real glsl_f32(T v) { return (ct_real)v; }

// ---------------------------------------------------------------------------
// vector types
#define GLSL_VEC2_BODY(VT, T)                                                   \
  T x, y;                                                                       \
  VT() : x(0), y(0) {}                                                          \
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0> \
  explicit VT(A s) : x(cvt(s)), y(cvt(s)) {}                                    \
  template <class A, class B> VT(A a, B b) : x(cvt(a)), y(cvt(b)) {}            \
  T &operator[](int i) { return i == 0 ? x : y; }                               \
  T operator[](int i) const { return i == 0 ? x : y; }                          \
  VT xy() const { return *this; }

template <class V> concept GlslVec2 = requires(V v) { v.x; v.y; } && !requires(V v) { v.z; };
template <class V> concept GlslVec3 = requires(V v) { v.x; v.y; v.z; } && !requires(V v) { v.w; };
template <class V> concept GlslVecWide2 = requires(V v) { v.z; };   // truncation to 2 components
template <class V> concept GlslVecWide3 = requires(V v) { v.w; };   // truncation to 3 components

template <class T> struct glsl_cvt {
  template <class A> static T c(A a) {
    if constexpr (std::is_same<T, uint32_t>::value) return glsl_u32(a);
    else if constexpr (std::is_same<T, int32_t>::value) return glsl_i32(a);
    else return (T)a;
  }
};

struct vec2 { static ct_real cvt(auto a) { return glsl_cvt<ct_real>::c(a); } GLSL_VEC2_BODY(vec2, ct_real)
  template <GlslVec2 V> vec2(const V &v) : x(cvt(v.x)), y(cvt(v.y)) {}
  template <GlslVecWide2 V> explicit vec2(const V &v) : x(cvt(v.x)), y(cvt(v.y)) {} };
struct ivec2 { static int32_t cvt(auto a) { return glsl_cvt<int32_t>::c(a); } GLSL_VEC2_BODY(ivec2, int32_t)
  template <GlslVec2 V> ivec2(const V &v) : x(cvt(v.x)), y(cvt(v.y)) {}
  template <GlslVecWide2 V> explicit ivec2(const V &v) : x(cvt(v.x)), y(cvt(v.y)) {} };
struct uvec2 { static uint32_t cvt(auto a) { return glsl_cvt<uint32_t>::c(a); } GLSL_VEC2_BODY(uvec2, uint32_t)
  template <GlslVec2 V> uvec2(const V &v) : x(cvt(v.x)), y(cvt(v.y)) {}
  template <GlslVecWide2 V> explicit uvec2(const V &v) : x(cvt(v.x)), y(cvt(v.y)) {} };
struct bvec2 { bool x, y; bvec2() : x(false), y(false) {} bvec2(bool a, bool b) : x(a), y(b) {} };

#define GLSL_VEC3_BODY(VT, V2, T)                                               \
  T x, y, z;                                                                    \
  VT() : x(0), y(0), z(0) {}                                                    \
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0> \
  explicit VT(A s) : x(cvt(s)), y(cvt(s)), z(cvt(s)) {}                         \
  template <class A, class B, class C> VT(A a, B b, C c) : x(cvt(a)), y(cvt(b)), z(cvt(c)) {} \
  template <class B> VT(const V2 &a, B b) : x(a.x), y(a.y), z(cvt(b)) {}        \
  T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }                \
  T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }           \
  V2 xy() const { return V2(x, y); }                                            \
  V2 yz() const { return V2(y, z); }                                            \
  V2 zx() const { return V2(z, x); }                                            \
  VT xyz() const { return *this; }

struct vec3 { static ct_real cvt(auto a) { return glsl_cvt<ct_real>::c(a); } GLSL_VEC3_BODY(vec3, vec2, ct_real)
  template <GlslVec3 V> vec3(const V &v) : x(cvt(v.x)), y(cvt(v.y)), z(cvt(v.z)) {}
  template <GlslVecWide3 V> explicit vec3(const V &v) : x(cvt(v.x)), y(cvt(v.y)), z(cvt(v.z)) {} };
struct ivec3 { static int32_t cvt(auto a) { return glsl_cvt<int32_t>::c(a); } GLSL_VEC3_BODY(ivec3, ivec2, int32_t)
  template <GlslVec3 V> ivec3(const V &v) : x(cvt(v.x)), y(cvt(v.y)), z(cvt(v.z)) {}
  template <GlslVecWide3 V> explicit ivec3(const V &v) : x(cvt(v.x)), y(cvt(v.y)), z(cvt(v.z)) {} };
struct uvec3 { static uint32_t cvt(auto a) { return glsl_cvt<uint32_t>::c(a); } GLSL_VEC3_BODY(uvec3, uvec2, uint32_t)
  template <GlslVec3 V> uvec3(const V &v) : x(cvt(v.x)), y(cvt(v.y)), z(cvt(v.z)) {}
  template <GlslVecWide3 V> explicit uvec3(const V &v) : x(cvt(v.x)), y(cvt(v.y)), z(cvt(v.z)) {} };
struct bvec3 { bool x, y, z; bvec3() : x(false), y(false), z(false) {} bvec3(bool a, bool b, bool c) : x(a), y(b), z(c) {} };

struct vec4 {
  ct_real x, y, z, w;
  static ct_real cvt(auto a) { return (ct_real)a; }
  vec4() : x(0), y(0), z(0), w(0) {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  explicit vec4(A s) : x(cvt(s)), y(cvt(s)), z(cvt(s)), w(cvt(s)) {}
  template <class A, class B, class C, class D> vec4(A a, B b, C c, D d) : x(cvt(a)), y(cvt(b)), z(cvt(c)), w(cvt(d)) {}
  template <class B> vec4(const vec3 &a, B b) : x(a.x), y(a.y), z(a.z), w(cvt(b)) {}
  ct_real &operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  ct_real operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  vec2 xy() const { return vec2(x, y); }
  vec3 xyz() const { return vec3(x, y, z); }
};
struct bvec4 { bool x, y, z, w; };

// ---------------------------------------------------------------------------
// component-wise operators
#define GLSL_BINOP2(VT, OP)                                                        \
  static inline VT operator OP(const VT &a, const VT &b) { return VT(a.x OP b.x, a.y OP b.y); } \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT operator OP(const VT &a, S s) { return VT(a.x OP s, a.y OP s); }           \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT operator OP(S s, const VT &a) { return VT(s OP a.x, s OP a.y); }           \
  static inline VT &operator OP##=(VT &a, const VT &b) { a = a OP b; return a; }              \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT &operator OP##=(VT &a, S s) { a = a OP s; return a; }
#define GLSL_BINOP3(VT, OP)                                                        \
  static inline VT operator OP(const VT &a, const VT &b) { return VT(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT operator OP(const VT &a, S s) { return VT(a.x OP s, a.y OP s, a.z OP s); } \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT operator OP(S s, const VT &a) { return VT(s OP a.x, s OP a.y, s OP a.z); } \
  static inline VT &operator OP##=(VT &a, const VT &b) { a = a OP b; return a; }              \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT &operator OP##=(VT &a, S s) { a = a OP s; return a; }
#define GLSL_BINOP4(VT, OP)                                                        \
  static inline VT operator OP(const VT &a, const VT &b) { return VT(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); } \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT operator OP(const VT &a, S s) { return VT(a.x OP s, a.y OP s, a.z OP s, a.w OP s); } \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT operator OP(S s, const VT &a) { return VT(s OP a.x, s OP a.y, s OP a.z, s OP a.w); } \
  static inline VT &operator OP##=(VT &a, const VT &b) { a = a OP b; return a; }              \
  template <class S, typename std::enable_if<std::is_arithmetic<S>::value, int>::type = 0> \
  static inline VT &operator OP##=(VT &a, S s) { a = a OP s; return a; }

// Scalar operands are converted to the vector's component type first, as the
// GLSL implicit conversions do (vec * double literal must stay single precision).
template <class VT, class S> static inline auto glsl_comp(S s) { return (decltype(VT::cvt(0)))s; }

GLSL_BINOP2(vec2, +) GLSL_BINOP2(vec2, -) GLSL_BINOP2(vec2, *) GLSL_BINOP2(vec2, /)
GLSL_BINOP2(ivec2, +) GLSL_BINOP2(ivec2, -) GLSL_BINOP2(ivec2, *) GLSL_BINOP2(ivec2, /)
GLSL_BINOP2(uvec2, +) GLSL_BINOP2(uvec2, -) GLSL_BINOP2(uvec2, *) GLSL_BINOP2(uvec2, /)
GLSL_BINOP3(vec3, +) GLSL_BINOP3(vec3, -) GLSL_BINOP3(vec3, *) GLSL_BINOP3(vec3, /)
GLSL_BINOP3(ivec3, +) GLSL_BINOP3(ivec3, -) GLSL_BINOP3(ivec3, *) GLSL_BINOP3(ivec3, /)
GLSL_BINOP3(uvec3, +) GLSL_BINOP3(uvec3, -) GLSL_BINOP3(uvec3, *) GLSL_BINOP3(uvec3, /)
GLSL_BINOP4(vec4, +) GLSL_BINOP4(vec4, -) GLSL_BINOP4(vec4, *) GLSL_BINOP4(vec4, /)

static inline vec2 operator-(const vec2 &a) { return vec2(-a.x, -a.y); }
static inline vec3 operator-(const vec3 &a) { return vec3(-a.x, -a.y, -a.z); }
static inline vec4 operator-(const vec4 &a) { return vec4(-a.x, -a.y, -a.z, -a.w); }
static inline ivec2 operator-(const ivec2 &a) { return ivec2(-a.x, -a.y); }
static inline ivec3 operator-(const ivec3 &a) { return ivec3(-a.x, -a.y, -a.z); }

// ---------------------------------------------------------------------------
// matrices (column major, as GLSL)
struct mat3 {
  vec3 c[3];
  mat3() {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  explicit mat3(A d) { c[0] = vec3((ct_real)d, 0.f, 0.f); c[1] = vec3(0.f, (ct_real)d, 0.f); c[2] = vec3(0.f, 0.f, (ct_real)d); }
  template <class... A, typename std::enable_if<sizeof...(A) == 9, int>::type = 0>
  mat3(A... a) { ct_real f[9] = {(ct_real)a...}; for (int i = 0; i < 3; i++) c[i] = vec3(f[3 * i], f[3 * i + 1], f[3 * i + 2]); }
  vec3 &operator[](int i) { return c[i]; }
  const vec3 &operator[](int i) const { return c[i]; }
};
struct mat4x3 {  // four columns of three rows (gl_ObjectToWorldEXT)
  vec3 c[4];
  vec3 &operator[](int i) { return c[i]; }
  const vec3 &operator[](int i) const { return c[i]; }
};

// flattening helper for mat4 constructors mixing vectors and scalars
struct glsl_flat {
  ct_real f[16]; int n = 0;
  void push(ct_real v) { f[n++] = v; }
  template <class A> typename std::enable_if<std::is_arithmetic<A>::value>::type add(A a) { push((ct_real)a); }
  void add(const vec3 &v) { push(v.x); push(v.y); push(v.z); }
  void add(const vec4 &v) { push(v.x); push(v.y); push(v.z); push(v.w); }
};
struct mat4 {
  vec4 c[4];
  mat4() {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  explicit mat4(A d) { for (int i = 0; i < 4; i++) { c[i] = vec4(0.f); c[i][i] = (ct_real)d; } }
  template <class A0, class A1, class... A>
  mat4(A0 a0, A1 a1, A... a) {
    glsl_flat fl; fl.add(a0); fl.add(a1); (fl.add(a), ...);
    for (int i = 0; i < 4; i++) c[i] = vec4(fl.f[4 * i], fl.f[4 * i + 1], fl.f[4 * i + 2], fl.f[4 * i + 3]);
  }
  vec4 &operator[](int i) { return c[i]; }
  const vec4 &operator[](int i) const { return c[i]; }
};

static inline ct_real dot(const vec2 &a, const vec2 &b) { return a.x * b.x + a.y * b.y; }
static inline ct_real dot(const vec3 &a, const vec3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline ct_real dot(const vec4 &a, const vec4 &b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

static inline vec3 operator*(const mat3 &m, const vec3 &v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }
static inline vec3 operator*(const vec3 &v, const mat3 &m) { return vec3(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])); }
static inline vec4 operator*(const mat4 &m, const vec4 &v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w; }
static inline vec4 operator*(const vec4 &v, const mat4 &m) { return vec4(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2]), dot(v, m.c[3])); }
static inline mat4 operator*(const mat4 &a, const mat4 &b) { mat4 r; for (int i = 0; i < 4; i++) r.c[i] = a * b.c[i]; return r; }
static inline mat3 operator*(const mat3 &a, const mat3 &b) { mat3 r; for (int i = 0; i < 3; i++) r.c[i] = a * b.c[i]; return r; }

static inline mat4 transpose(const mat4 &m) {
  mat4 r;
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) r.c[i][j] = m.c[j][i];
  return r;
}

// Inverse by cofactor expansion (m[col][row]).  The CUDA kernels use the same
// sequence of operations.
static inline mat4 inverse(const mat4 &M) {
  ct_real m[16];
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) m[4 * i + j] = M.c[i][j];
  ct_real inv[16];
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
  ct_real det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  mat4 R;
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) R.c[i][j] = inv[4 * i + j] / det;
  return R;
}

// ---------------------------------------------------------------------------
// built-in functions
template <class A, class B> static inline auto glsl_common(A a, B b) {
  if constexpr (std::is_floating_point<A>::value || std::is_floating_point<B>::value) return (ct_real)0;
  else if constexpr (std::is_unsigned<A>::value || std::is_unsigned<B>::value) return (uint32_t)0;
  else return (int32_t)0;
}
template <class A, class B, typename std::enable_if<std::is_arithmetic<A>::value && std::is_arithmetic<B>::value, int>::type = 0>
static inline auto min(A a, B b) { using T = decltype(glsl_common(a, b)); T x = (T)a, y = (T)b; return y < x ? y : x; }
template <class A, class B, typename std::enable_if<std::is_arithmetic<A>::value && std::is_arithmetic<B>::value, int>::type = 0>
static inline auto max(A a, B b) { using T = decltype(glsl_common(a, b)); T x = (T)a, y = (T)b; return x < y ? y : x; }
template <class A, class B, class C, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
static inline auto clamp(A x, B lo, C hi) { return min(max(x, lo), hi); }
static inline vec3 min(const vec3 &a, const vec3 &b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
static inline vec3 max(const vec3 &a, const vec3 &b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
template <class S> static inline vec3 min(const vec3 &a, S b) { return min(a, vec3((ct_real)b)); }
template <class S> static inline vec3 max(const vec3 &a, S b) { return max(a, vec3((ct_real)b)); }
template <class S> static inline vec3 min(S b, const vec3 &a) { return min(vec3((ct_real)b), a); }
template <class S, class T> static inline vec3 clamp(const vec3 &x, S lo, T hi) { return min(max(x, lo), hi); }

template <class A, class B, class C, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
static inline ct_real mix(A x, B y, C a) { ct_real fx = (ct_real)x, fy = (ct_real)y, fa = (ct_real)a; return fx * (1.0f - fa) + fy * fa; }
template <class C> static inline vec3 mix(const vec3 &x, const vec3 &y, C a) { ct_real fa = (ct_real)a; return x * (1.0f - fa) + y * fa; }
template <class C> static inline vec4 mix(const vec4 &x, const vec4 &y, C a) { ct_real fa = (ct_real)a; return x * (1.0f - fa) + y * fa; }
static inline vec4 mix(const vec4 &x, const vec4 &y, const bvec4 &a) {
  return vec4(a.x ? y.x : x.x, a.y ? y.y : x.y, a.z ? y.z : x.z, a.w ? y.w : x.w);
}

static inline ct_real sign(ct_real x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
static inline vec3 sign(const vec3 &v) { return vec3(sign(v.x), sign(v.y), sign(v.z)); }
using std::abs;
static inline vec2 abs(const vec2 &v) { return vec2(std::fabs(v.x), std::fabs(v.y)); }
static inline vec3 abs(const vec3 &v) { return vec3(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }
static inline ct_real length(const vec3 &v) { return std::sqrt(dot(v, v)); }
static inline ct_real length(const vec2 &v) { return std::sqrt(dot(v, v)); }
static inline vec3 normalize(const vec3 &v) { ct_real l = length(v); return vec3(v.x / l, v.y / l, v.z / l); }
static inline ct_real distance(const vec3 &a, const vec3 &b) { return length(a - b); }
static inline vec3 cross(const vec3 &a, const vec3 &b) {
  return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
#ifdef CT_ORACLE_FP64
// double precision: the C library's functions
using std::sqrt;
using std::exp;
using std::floor;
using std::isnan;
using std::isinf;
using std::pow;
using std::cos;
using std::sin;
static inline vec3 pow(const vec3 &a, const vec3 &b) { return vec3(std::pow(a.x, b.x), std::pow(a.y, b.y), std::pow(a.z, b.z)); }
static inline vec4 pow(const vec4 &a, const vec4 &b) { return vec4(std::pow(a.x, b.x), std::pow(a.y, b.y), std::pow(a.z, b.z), std::pow(a.w, b.w)); }
static inline double fract(double x) { return x - std::floor(x); }
#else
static inline float sqrt(float x) { return std::sqrt(x); }
// GLSL leaves the precision of pow, sin and cos to the implementation.  The
// shim takes the ones of cube-tracing_b200/csrc/ct_fpmath.h, which the CUDA
// kernels call too, so that scatter directions (random_cosine_direction,
// prng.glsl:84-106) and the dielectric reflectance (prng.glsl:214-218) come
// out bit-identical on both sides.
static inline float pow(float a, float b) { return ct_powf(a, b); }
static inline vec3 pow(const vec3 &a, const vec3 &b) { return vec3(ct_powf(a.x, b.x), ct_powf(a.y, b.y), ct_powf(a.z, b.z)); }
static inline vec4 pow(const vec4 &a, const vec4 &b) { return vec4(ct_powf(a.x, b.x), ct_powf(a.y, b.y), ct_powf(a.z, b.z), ct_powf(a.w, b.w)); }
static inline float exp(float x) { return std::exp(x); }
static inline float cos(float x) { return ct_cosf(x); }
static inline float sin(float x) { return ct_sinf(x); }
static inline float floor(float x) { return std::floor(x); }
static inline float fract(float x) { return x - std::floor(x); }

static inline bool isnan(float x) { return std::isnan(x); }
static inline bool isinf(float x) { return std::isinf(x); }
#endif
static inline bvec3 isnan(const vec3 &v) { return bvec3(std::isnan(v.x), std::isnan(v.y), std::isnan(v.z)); }
static inline bvec3 isinf(const vec3 &v) { return bvec3(std::isinf(v.x), std::isinf(v.y), std::isinf(v.z)); }
static inline bool any(const bvec3 &b) { return b.x || b.y || b.z; }
static inline bool all(const bvec3 &b) { return b.x && b.y && b.z; }
static inline bool any(const bvec2 &b) { return b.x || b.y; }
static inline bool all(const bvec2 &b) { return b.x && b.y; }
static inline bvec3 lessThan(const vec3 &a, const vec3 &b) { return bvec3(a.x < b.x, a.y < b.y, a.z < b.z); }
static inline bvec2 lessThan(const vec2 &a, const vec2 &b) { return bvec2(a.x < b.x, a.y < b.y); }
static inline bvec2 lessThan(const ivec2 &a, const ivec2 &b) { return bvec2(a.x < b.x, a.y < b.y); }
static inline bvec4 lessThan(const vec4 &a, const vec4 &b) { return bvec4{a.x < b.x, a.y < b.y, a.z < b.z, a.w < b.w}; }
static inline bvec3 lessThanEqual(const vec3 &a, const vec3 &b) { return bvec3(a.x <= b.x, a.y <= b.y, a.z <= b.z); }
static inline bvec3 greaterThan(const vec3 &a, const vec3 &b) { return bvec3(a.x > b.x, a.y > b.y, a.z > b.z); }
static inline bvec2 greaterThanEqual(const ivec2 &a, const ivec2 &b) { return bvec2(a.x >= b.x, a.y >= b.y); }
static inline bvec3 equal(const vec3 &a, const vec3 &b) { return bvec3(a.x == b.x, a.y == b.y, a.z == b.z); }
static inline bvec2 equal(const ivec2 &a, const ivec2 &b) { return bvec2(a.x == b.x, a.y == b.y); }
static inline bvec3 notEqual(const vec3 &a, const vec3 &b) { return bvec3(a.x != b.x, a.y != b.y, a.z != b.z); }

static inline int32_t floatBitsToInt(ct_real r) { float f = (float)r; int32_t i; std::memcpy(&i, &f, 4); return i; }
static inline float intBitsToFloat(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline uint32_t atomicAdd(uint32_t &a, uint32_t v) { uint32_t o = a; a += v; return o; }
static inline uint32_t atomicOr(uint32_t &a, uint32_t v) { uint32_t o = a; a |= v; return o; }

// ---------------------------------------------------------------------------
// Daxa type names (daxa/daxa.inl maps these onto the GLSL types)
typedef uint32_t daxa_b32;  // 4 bytes, as in Daxa's buffer layouts
typedef uint32_t daxa_u32;
typedef int32_t daxa_i32;
typedef uint64_t daxa_u64;
typedef ct_real daxa_f32;
typedef vec2 daxa_f32vec2;
typedef vec3 daxa_f32vec3;
typedef vec4 daxa_f32vec4;
typedef ivec2 daxa_i32vec2;
typedef ivec3 daxa_i32vec3;
typedef uvec2 daxa_u32vec2;
typedef uvec3 daxa_u32vec3;
typedef mat3 daxa_f32mat3x3;
typedef mat4 daxa_f32mat4x4;
typedef mat4x3 daxa_f32mat4x3;

// Headless images: RGBA32F, row major.
struct glsl_image { uint32_t width, height; vec4 *texels; };
typedef glsl_image *daxa_ImageViewId;
typedef uint64_t daxa_SamplerId;
static inline glsl_image &daxa_image2D(daxa_ImageViewId id) { return *id; }
static inline void imageStore(glsl_image &img, ivec2 p, const vec4 &v) { img.texels[(size_t)p.y * img.width + p.x] = v; }
static inline vec4 imageLoad(glsl_image &img, ivec2 p) { return img.texels[(size_t)p.y * img.width + p.x]; }

// acceleration structures (opaque to the shaders)
struct OracleAccel;
typedef const OracleAccel *daxa_TlasId;
static inline daxa_TlasId daxa_accelerationStructureEXT(daxa_TlasId t) { return t; }

#define daxa_BufferPtr(T) T *
#define daxa_RWBufferPtr(T) T *
#define DAXA_DECL_BUFFER_PTR(T)
#define deref(x) (*(x))
#define DAXA_DECL_PUSH_CONSTANT(T, NAME)

// buffer_reference blocks, produced by the source transform from
// `layout(buffer_reference, scalar) buffer NAME {T field[]; };`
#define GLSL_BUFREF_ARRAY(NAME, T, FIELD)                                     \
  struct NAME { T *FIELD; explicit NAME(uint64_t a) : FIELD((T *)(uintptr_t)a) {} };
#define GLSL_BUFREF_ONE(NAME, T, FIELD)                                       \
  struct NAME { T &FIELD; explicit NAME(uint64_t a) : FIELD(*(T *)(uintptr_t)a) {} };

// ---------------------------------------------------------------------------
// ray tracing built-ins (values set by the oracle's pipeline emulation)
#define gl_RayFlagsNoneEXT 0u
#define gl_RayFlagsOpaqueEXT 1u
#define gl_RayFlagsTerminateOnFirstHitEXT 4u
#define gl_RayQueryCandidateIntersectionAABBEXT 1u
#define gl_RayQueryCommittedIntersectionNoneEXT 0u
#define gl_RayQueryCommittedIntersectionGeneratedEXT 2u

extern thread_local uvec3 gl_LaunchIDEXT;
extern thread_local uvec3 gl_LaunchSizeEXT;
extern thread_local uvec3 gl_GlobalInvocationID;
extern thread_local uvec3 gl_NumWorkGroups;
extern thread_local vec3 gl_WorldRayOriginEXT;
extern thread_local vec3 gl_WorldRayDirectionEXT;
extern thread_local mat4x3 gl_ObjectToWorldEXT;
extern thread_local int32_t gl_InstanceCustomIndexEXT;
extern thread_local int32_t gl_PrimitiveID;
extern thread_local ct_real gl_HitTEXT;

bool reportIntersectionEXT(ct_real t, uint32_t kind);
void executeCallableEXT(uint32_t sbt_index, uint32_t location);
void traceRayEXT(daxa_TlasId tlas, uint32_t flags, uint32_t cull, uint32_t sbt_offset, uint32_t sbt_stride,
                 uint32_t miss_index, vec3 origin, ct_real tmin, vec3 dir, ct_real tmax, int payload);

struct rayQueryEXT {
  daxa_TlasId tlas;
  uint32_t flags;
  vec3 origin, dir;
  ct_real tmin, tmax;
  // candidate list prepared at initialisation, presented in order
  uint32_t *cand;      // packed (instance << 27 | primitive) is not enough; two arrays
  uint32_t *cand_inst;
  uint32_t n, cap, next, cur;
  bool committed;
  ct_real committed_t;
  bool terminated;
  rayQueryEXT() : cand(nullptr), cand_inst(nullptr), n(0), cap(0), next(0), cur(0), committed(false), committed_t(0), terminated(false) {}
  ~rayQueryEXT();
  rayQueryEXT(const rayQueryEXT &) = delete;
};
void rayQueryInitializeEXT(rayQueryEXT &q, daxa_TlasId tlas, uint32_t flags, uint32_t cull, vec3 origin, ct_real tmin, vec3 dir, ct_real tmax);
bool rayQueryProceedEXT(rayQueryEXT &q);
uint32_t rayQueryGetIntersectionTypeEXT(rayQueryEXT &q, bool committed);
int32_t rayQueryGetIntersectionInstanceCustomIndexEXT(rayQueryEXT &q, bool committed);
int32_t rayQueryGetIntersectionPrimitiveIndexEXT(rayQueryEXT &q, bool committed);
void rayQueryGenerateIntersectionEXT(rayQueryEXT &q, ct_real t);
void rayQueryTerminateEXT(rayQueryEXT &q);
