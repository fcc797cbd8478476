// Shared device helpers for the T-matrix kernels (sm_100a, FP64 throughout).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "tmx_internal.h"

// complex numbers are double2 (x = re, y = im)
typedef double2 cplx;

__host__ __device__ __forceinline__ cplx mkc(double re, double im) {
  return make_double2(re, im);
}
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) {
  return mkc(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) {
  return mkc(a.x - b.x, a.y - b.y);
}
// (a.x + i a.y)(b.x + i b.y) in the textbook order (ac - bd, ad + bc)
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) {
  return mkc(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ double cnorm2(cplx a) {
  return a.x * a.x + a.y * a.y;
}

// Complex quotient (a + ib)/(c + id) by Smith's algorithm (R. L. Smith,
// "Algorithm 116: Complex division", CACM 5(8), 1962): scale by the larger of
// |c| and |d| so that no intermediate squares the divisor.
__host__ __device__ __forceinline__ cplx cdiv(cplx num, cplx den) {
  const double a = num.x, b = num.y, c = den.x, d = den.y;
  if (fabs(c) < fabs(d)) {
    const double r = c / d;
    const double t = c * r + d;
    return mkc((a * r + b) / t, (b * r - a) / t);
  }
  const double r = d / c;
  const double t = d * r + c;
  return mkc((b * r + a) / t, (b - a * r) / t);
}

// 1 / z as the complex quotient (1 + 0i) / z
__host__ __device__ __forceinline__ cplx cinv(cplx z) {
  return cdiv(mkc(1., 0.), z);
}

// bounded spin helper: device loops that wait never spin forever
#define TMX_SPIN_LIMIT (1u << 26)
