/*
 * detmath.h -- deterministic transcendental functions for host and device.
 *
 * The WGSL passes call exp, pow, sin and cos.  Their results on the GPU
 * differ between vendors and from libm on the host, which would make a
 * bit-exact CPU/GPU comparison impossible.  Every function here is written
 * from the mathematics (Cody & Waite argument reduction, "Software Manual for
 * the Elementary Functions", 1980, plus truncated Taylor / atanh series) and
 * evaluated in IEEE binary64 with a fixed operation order, then rounded once
 * to binary32.  Compiled without FMA contraction (host: -ffp-contract=off,
 * device: -fmad=false) both sides produce identical bits; the relative error
 * of every float result is below 1 ulp (checked in tests/test_detmath.py).
 */
#ifndef VXE_DETMATH_H
#define VXE_DETMATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define VXE_HD __host__ __device__ __forceinline__
/* Out of line on the device: called from dozens of sites, inlining them all
 * overflows the instruction cache of the frame kernels. */
#define VXE_HD_CALL __host__ __device__ __noinline__
#else
#define VXE_HD static inline
#define VXE_HD_CALL static inline
#include <string.h>
#endif

/* pi/2 split into three binary64 pieces; the first two carry 33 significant
 * bits so k * piece is exact for |k| < 2^20 (derived from 80 decimal digits). */
#define VXE_PIO2_1 1.5707963267341256
#define VXE_PIO2_2 6.077100506303966e-11
#define VXE_PIO2_3 2.0222662487959506e-21
#define VXE_TWO_OVER_PI 0.6366197723675814
/* ln 2 split, first piece with 32 significant bits. */
#define VXE_LN2_1 0.6931471803691238
#define VXE_LN2_2 1.9082149292705877e-10
#define VXE_LOG2E 1.4426950408889634
#define VXE_LN2 0.6931471805599453

VXE_HD uint64_t vxe_d2u(double d) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  memcpy(&u, &d, sizeof(u));
  return u;
#endif
}

VXE_HD double vxe_u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, sizeof(d));
  return d;
#endif
}

VXE_HD double vxe_floor_d(double x) {
#if defined(__CUDA_ARCH__)
  return floor(x);
#else
  return __builtin_floor(x);
#endif
}

/* 2^k for integer k in [-1022, 1023] built from its bit pattern. */
VXE_HD double vxe_pow2i(int k) { return vxe_u2d((uint64_t)(int64_t)(k + 1023) << 52); }

/* e^x in binary64 (|x| <= 745 handled; beyond returns inf / 0). */
VXE_HD double vxe_exp_d(double x) {
  if (x != x) return x;
  if (x > 709.0) return vxe_u2d(0x7FF0000000000000ull);
  if (x < -745.0) return 0.0;
  const double kd = vxe_floor_d(x * VXE_LOG2E + 0.5);
  const int k = (int)kd;
  const double r = (x - kd * VXE_LN2_1) - kd * VXE_LN2_2; /* |r| <= 0.3466 */
  /* Taylor series of e^r to degree 12, Horner form. */
  double p = 2.08767569878681e-09;
  p = p * r + 2.505210838544172e-08;
  p = p * r + 2.755731922398589e-07;
  p = p * r + 2.7557319223985893e-06;
  p = p * r + 2.48015873015873e-05;
  p = p * r + 0.0001984126984126984;
  p = p * r + 0.001388888888888889;
  p = p * r + 0.008333333333333333;
  p = p * r + 0.041666666666666664;
  p = p * r + 0.16666666666666666;
  p = p * r + 0.5;
  p = p * r + 1.0;
  p = p * r + 1.0;
  if (k < -1000) return (p * vxe_pow2i(k + 200)) * vxe_pow2i(-200);
  return p * vxe_pow2i(k);
}

/* Natural log in binary64 for x > 0 (0 -> -inf, x < 0 or NaN -> NaN). */
VXE_HD double vxe_log_d(double x) {
  if (x != x || x < 0.0) return vxe_u2d(0x7FF8000000000000ull);
  if (x == 0.0) return vxe_u2d(0xFFF0000000000000ull);
  if (x == vxe_u2d(0x7FF0000000000000ull)) return x;
  uint64_t u = vxe_d2u(x);
  int e = (int)((u >> 52) & 0x7FF);
  if (e == 0) { /* subnormal binary64: normalise */
    x = x * 18014398509481984.0; /* 2^54 */
    u = vxe_d2u(x);
    e = (int)((u >> 52) & 0x7FF) - 54;
  }
  e -= 1023;
  double m = vxe_u2d((u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull); /* [1,2) */
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  /* log m = 2 atanh(s), s = (m-1)/(m+1), |s| <= 0.1716 */
  const double s = (m - 1.0) / (m + 1.0);
  const double s2 = s * s;
  double q = 1.0 / 19.0;
  q = q * s2 + 1.0 / 17.0;
  q = q * s2 + 1.0 / 15.0;
  q = q * s2 + 1.0 / 13.0;
  q = q * s2 + 1.0 / 11.0;
  q = q * s2 + 1.0 / 9.0;
  q = q * s2 + 1.0 / 7.0;
  q = q * s2 + 1.0 / 5.0;
  q = q * s2 + 1.0 / 3.0;
  q = q * s2 + 1.0;
  const double lm = 2.0 * s * q;
  const double ed = (double)e;
  return (ed * VXE_LN2_1 + lm) + ed * VXE_LN2_2;
}

/* sin / cos of r for |r| <= pi/4 (Taylor to degree 15 / 16). */
VXE_HD double vxe_sin_poly(double r) {
  const double r2 = r * r;
  double p = -7.647163731819816e-13;
  p = p * r2 + 1.6059043836821613e-10;
  p = p * r2 - 2.505210838544172e-08;
  p = p * r2 + 2.755731922398589e-06;
  p = p * r2 - 0.0001984126984126984;
  p = p * r2 + 0.008333333333333333;
  p = p * r2 - 0.16666666666666666;
  return r + r * (r2 * p);
}

VXE_HD double vxe_cos_poly(double r) {
  const double r2 = r * r;
  double p = 4.779477332387385e-14;
  p = p * r2 - 1.1470745597729725e-11;
  p = p * r2 + 2.08767569878681e-09;
  p = p * r2 - 2.755731922398589e-07;
  p = p * r2 + 2.48015873015873e-05;
  p = p * r2 - 0.001388888888888889;
  p = p * r2 + 0.041666666666666664;
  p = p * r2 - 0.5;
  return 1.0 + r2 * p;
}

/* Reduce x to r in [-pi/4, pi/4] and quadrant q = k mod 4. */
VXE_HD double vxe_reduce_pio2(double x, int* q) {
  const double kd = vxe_floor_d(x * VXE_TWO_OVER_PI + 0.5);
  *q = (int)((int64_t)kd & 3);
  return ((x - kd * VXE_PIO2_1) - kd * VXE_PIO2_2) - kd * VXE_PIO2_3;
}

VXE_HD_CALL float vxe_sinf(float xf) {
  const double x = (double)xf;
  if (x != x || x - x != 0.0) return (float)(x - x); /* NaN for NaN / inf */
  if (x > 1e18 || x < -1e18) return 0.0f;              /* beyond the reduction */
  int q;
  const double r = vxe_reduce_pio2(x, &q);
  double v;
  if (q == 0) v = vxe_sin_poly(r);
  else if (q == 1) v = vxe_cos_poly(r);
  else if (q == 2) v = -vxe_sin_poly(r);
  else v = -vxe_cos_poly(r);
  return (float)v;
}

VXE_HD_CALL float vxe_cosf(float xf) {
  const double x = (double)xf;
  if (x != x || x - x != 0.0) return (float)(x - x);
  if (x > 1e18 || x < -1e18) return 1.0f;
  int q;
  const double r = vxe_reduce_pio2(x, &q);
  double v;
  if (q == 0) v = vxe_cos_poly(r);
  else if (q == 1) v = -vxe_sin_poly(r);
  else if (q == 2) v = -vxe_cos_poly(r);
  else v = vxe_sin_poly(r);
  return (float)v;
}

VXE_HD_CALL float vxe_expf(float x) { return (float)vxe_exp_d((double)x); }

/* pow for the non-negative bases the passes use: pow(0, y>0) = 0,
 * pow(x, 0) = 1, negative bases give NaN (WGSL leaves them undefined). */
VXE_HD_CALL float vxe_powf(float x, float y) {
  if (y == 0.0f) return 1.0f;
  if (x == 0.0f) return y > 0.0f ? 0.0f : vxe_u2d(0x7FF0000000000000ull);
  if (x == 1.0f) return 1.0f;
  return (float)vxe_exp_d((double)y * vxe_log_d((double)x));
}

#endif /* VXE_DETMATH_H */
