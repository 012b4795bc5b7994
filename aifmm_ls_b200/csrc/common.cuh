// common.cuh -- shared device helpers for the AIFMM-LS B200 solver.
//
// Complex numbers are double2 (x = real, y = imaginary); matrices are
// column-major with an explicit leading dimension.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>

#define AIFMM_HD __host__ __device__ __forceinline__

AIFMM_HD double2 cmk(double re, double im) { return make_double2(re, im); }
AIFMM_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
AIFMM_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
AIFMM_HD double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
AIFMM_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
AIFMM_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// (a+bi)(c+di) = (ac-bd) + (ad+bc)i
AIFMM_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// conj(a) * b
AIFMM_HD double2 cmulc(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
AIFMM_HD double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
AIFMM_HD double cabsd(double2 a) { return hypot(a.x, a.y); }
// a / b (Smith's algorithm, as a compiler's complex division would do)
AIFMM_HD double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  double r = b.x / b.y, d = b.x * r + b.y;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
// c += a*b using fused multiply-adds
AIFMM_HD double2 cfma(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x); c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y); c.y = fma(a.y, b.x, c.y);
  return c;
}
// c += conj(a)*b
AIFMM_HD double2 cfmac(double2 a, double2 b, double2 c) {
  c.x = fma(a.x, b.x, c.x); c.x = fma(a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y); c.y = fma(-a.y, b.x, c.y);
  return c;
}

// The same operations on complex64 (float2), for the factorisation of the mixed
// form; the kernels that serve both forms are templates over the complex type.
AIFMM_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
AIFMM_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
AIFMM_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
AIFMM_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
AIFMM_HD float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
AIFMM_HD double cabsd(float2 a) { return hypot((double)a.x, (double)a.y); }
AIFMM_HD float2 cdiv(float2 a, float2 b) {
  if (fabsf(b.x) >= fabsf(b.y)) {
    float r = b.y / b.x, d = b.x + b.y * r;
    return make_float2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  float r = b.x / b.y, d = b.x * r + b.y;
  return make_float2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
AIFMM_HD float2 cfma(float2 a, float2 b, float2 c) {
  c.x = fmaf(a.x, b.x, c.x); c.x = fmaf(-a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y); c.y = fmaf(a.y, b.x, c.y);
  return c;
}
AIFMM_HD float2 cfmac(float2 a, float2 b, float2 c) {
  c.x = fmaf(a.x, b.x, c.x); c.x = fmaf(a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y); c.y = fmaf(-a.y, b.x, c.y);
  return c;
}

// Complex type traits: R the real type, mk(re, im), conversions to and from
// complex128 (round to nearest on the way down).
template <typename C> struct cplx;
template <> struct cplx<double2> {
  using R = double;
  AIFMM_HD static double2 mk(double re, double im) { return make_double2(re, im); }
  AIFMM_HD static double2 from(double2 v) { return v; }
  AIFMM_HD static double2 from(float2 v) { return make_double2(v.x, v.y); }
};
template <> struct cplx<float2> {
  using R = float;
  AIFMM_HD static float2 mk(double re, double im) { return make_float2((float)re, (float)im); }
  AIFMM_HD static float2 from(double2 v) { return make_float2((float)v.x, (float)v.y); }
  AIFMM_HD static float2 from(float2 v) { return v; }
};

// Contrast kinds: 0..5 are the reference's Qchoice values (LS/LS_functions.hpp:99-112),
// 10 = amp*exp(-width|x|^2), 11 = amp*[|x| < radius].
enum { Q_GAUSSIAN160 = 0, Q_MULTI_GAUSS = 1, Q_PLASMA = 2, Q_FLATBUMP = 3, Q_CAVITY = 4,
       Q_LENS = 5, Q_GAUSS_AW = 10, Q_DISK = 11 };

// Everything a matrix-entry evaluation needs (all device pointers).
struct EntryCtx {
  int rank;        // points per leaf (n_cheb^2)
  int depth;       // leaf level
  double kappa;
  const double2* pts;     // N grid points
  const double* q;        // contrast at the grid points
  const double2* leafc;   // leaf centres (Morton order)
  const int2* leafxy;     // leaf grid coordinates
  const double2* M;       // far-field coefficients, 121 x rank, column-major
  const double2* nearT;   // 9 near tables, rank x rank column-major each
};

#define AIFMM_CUDA_OK(call) ((call) == cudaSuccess)
