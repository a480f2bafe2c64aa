// ct_fpmath.h -- sine, cosine and integer powers with one fixed sequence of
// IEEE single-precision operations, so that every compiler that keeps the
// written order (nvcc --fmad=false, g++ -ffp-contract=off) gets the same
// bits.
//
// GLSL leaves the precision of sin, cos and pow to the implementation, and
// the shaders this library follows use them in the path tracer's scatter
// directions (random_cosine_direction, prng.glsl:84-106) and in the
// dielectric reflectance (prng.glsl:214-218).  The CUDA kernels call these
// functions there, and the CPU oracle's GLSL shim maps the shaders' sin, cos
// and pow to them, so both sides sample identical directions.
//
// Method:
//   * argument reduction x = k*pi/2 + r, |r| <= pi/4, after Cody and Waite
//     (1980): pi/2 split into three single-precision parts, the first two
//     with 12 significant bits so that k*P1 and k*P2 are exact for |k| < 2^12;
//   * sin r and cos r by their Taylor series through r^11 and r^12 (Horner
//     form; the first omitted terms are below 2e-9 relative on |r| <= pi/4);
//   * the quadrant k mod 4 selects and signs the two.
// Accurate to a few units in the last place for |x| < 2^12 (checked against
// double-precision sin/cos by the test suite); the path only needs [0, 2*pi).
//
// ct_powf: exact small integer exponents (|y| <= 32) by repeated
// multiplication from the left; other exponents through exp2(y*log2(x))
// of the platform's library (not reached by Lambertian scenes).
#pragma once

#if defined(__CUDACC__)
#define CT_FPM_FN __host__ __device__ __forceinline__
#include <cuda_runtime.h>
#else
#define CT_FPM_FN static inline
#include <cmath>
#endif

namespace ctfp {

CT_FPM_FN float floor_(float x) {
#if defined(__CUDA_ARCH__)
  return floorf(x);
#else
  return std::floor(x);
#endif
}

// sin(r), cos(r) for |r| <= pi/4
CT_FPM_FN float sin_poly(float r) {
  const float r2 = r * r;
  float p = -0x1.ae6456p-26f;
  p = p * r2 + 0x1.71de3ap-19f;
  p = p * r2 + -0x1.a01a02p-13f;
  p = p * r2 + 0x1.111112p-7f;
  p = p * r2 + -0x1.555556p-3f;
  return r + (r * r2) * p;
}
CT_FPM_FN float cos_poly(float r) {
  const float r2 = r * r;
  float p = 0x1.1eed8ep-29f;
  p = p * r2 + -0x1.27e4fcp-22f;
  p = p * r2 + 0x1.a01a02p-16f;
  p = p * r2 + -0x1.6c16c2p-10f;
  p = p * r2 + 0x1.555556p-5f;
  p = p * r2 + -0x1.0p-1f;
  return 1.0f + r2 * p;
}

// x = k*pi/2 + r; returns r, k mod 4 in *q
CT_FPM_FN float reduce(float x, int *q) {
  const float k = floor_(x * 0x1.45f306p-1f + 0.5f);
  float r = x - k * 0x1.92p+0f;
  r = r - k * 0x1.fb4p-12f;
  r = r - k * 0x1.4442d2p-24f;
  *q = ((int)k) & 3;
  return r;
}

}  // namespace ctfp

CT_FPM_FN float ct_sinf(float x) {
  int q;
  const float r = ctfp::reduce(x, &q);
  const float s = ctfp::sin_poly(r), c = ctfp::cos_poly(r);
  return q == 0 ? s : q == 1 ? c : q == 2 ? -s : -c;
}

CT_FPM_FN float ct_cosf(float x) {
  int q;
  const float r = ctfp::reduce(x, &q);
  const float s = ctfp::sin_poly(r), c = ctfp::cos_poly(r);
  return q == 0 ? c : q == 1 ? -s : q == 2 ? -c : s;
}

CT_FPM_FN float ct_powf(float x, float y) {
  if (y == ctfp::floor_(y) && y >= -32.0f && y <= 32.0f) {
    const int n = (int)(y < 0.0f ? -y : y);
    float p = 1.0f;
    for (int i = 0; i < n; i++) p = p * x;
    return y < 0.0f ? 1.0f / p : p;
  }
#if defined(__CUDA_ARCH__)
  return exp2f(y * log2f(x));
#else
  return std::exp2(y * std::log2(x));
#endif
}
