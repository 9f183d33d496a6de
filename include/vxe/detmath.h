/*
 * detmath.h -- deterministic transcendental functions for host and device.
 *
 * The WGSL passes call exp, pow, sin and cos.  Their results on the GPU
 * differ between vendors and from libm on the host, which would make a
 * bit-exact CPU/GPU comparison impossible.  Every function here is written
 * from the mathematics (Cody & Waite argument reduction, "Software Manual for
 * the Elementary Functions", 1980, plus truncated Taylor / atanh series) with a
 * fixed operation order.  Only correctly rounded IEEE operations are used:
 * +, -, *, /, and fused multiply-adds written out explicitly (vxe_fmaf:
 * one rounding on every machine).  Compiled without FMA contraction
 * (host: -ffp-contract=off, device: -fmad=false), both sides therefore produce
 * identical bits.
 *
 * exp, sin and cos are evaluated in binary32, with fused multiply-adds in the
 * argument reduction and in the Horner steps: exp within 1 ulp, sin and cos
 * within 1.5 ulp (8e-8 absolute near their zeros), inside WGSL's own bounds
 * for these builtins (exp 3 + 2|x| ulp, sin / cos 2^-11 absolute on [-pi, pi]).
 * sin and cos of |x| > 65536 use a binary64 reduction.  pow carries log x
 * and y log x as unevaluated binary32 pairs: within 1.25 ulp for exponents up
 * to 8, 3.5 ulp at 96 (the error grows with |y log x|).  The bounds are
 * checked in tests/test_detmath.py.
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

VXE_HD float vxe_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, sizeof(f));
  return f;
#endif
}

/* Fused multiply-adds (one rounding) and round-to-nearest-even; correctly
 * rounded on both sides. */
VXE_HD float vxe_fmaf(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return __builtin_fmaf(a, b, c);
#endif
}

VXE_HD float vxe_rintf(float x) {
#if defined(__CUDA_ARCH__)
  return rintf(x);
#else
  return __builtin_rintf(x);
#endif
}

/* 2^k for integer k in [-126, 127]. */
VXE_HD float vxe_pow2if(int k) { return vxe_u2f((uint32_t)(k + 127) << 23); }

VXE_HD uint32_t vxe_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, sizeof(u));
  return u;
#endif
}

/* 1/x correctly rounded in binary32. */
VXE_HD float vxe_rcpf(float x) {
#if defined(__CUDA_ARCH__)
  return __frcp_rn(x);
#else
  return 1.0f / x;
#endif
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

/* binary32 pi/2 split into three pieces (the first is pi/2 rounded to
 * binary32), for the fused reduction below. */
#define VXE_PIO2F_1 1.5707963705062866f
#define VXE_PIO2F_2 -4.371138828673793e-08f
#define VXE_PIO2F_3 -1.7151245100058819e-15f

/* x - k pi/2 for |x| <= 65536 (|k| < 2^16): every product enters a fused
 * multiply-add unrounded, so only the three sums round. */
VXE_HD float vxe_reduce_pio2f(float x, int* q) {
  const float kf = vxe_rintf(x * 0.6366197466850281f);
  *q = (int)kf & 3;
  float r = vxe_fmaf(-kf, VXE_PIO2F_1, x);
  r = vxe_fmaf(-kf, VXE_PIO2F_2, r);
  return vxe_fmaf(-kf, VXE_PIO2F_3, r);
}

/* sin r and cos r for |r| <= pi/4 (+ rounding): Taylor series to degree 11
 * and 12 (truncation below 2^-29), Horner form in r^2. */
VXE_HD float vxe_sin_polyf(float r) {
  const float s = r * r;
  float p = -1.0f / 39916800.0f;
  p = vxe_fmaf(p, s, 1.0f / 362880.0f);
  p = vxe_fmaf(p, s, -1.0f / 5040.0f);
  p = vxe_fmaf(p, s, 1.0f / 120.0f);
  p = vxe_fmaf(p, s, -1.0f / 6.0f);
  return vxe_fmaf(r * s, p, r);
}

VXE_HD float vxe_cos_polyf(float r) {
  const float s = r * r;
  float p = 1.0f / 479001600.0f;
  p = vxe_fmaf(p, s, -1.0f / 3628800.0f);
  p = vxe_fmaf(p, s, 1.0f / 40320.0f);
  p = vxe_fmaf(p, s, -1.0f / 720.0f);
  p = vxe_fmaf(p, s, 1.0f / 24.0f);
  p = vxe_fmaf(p, s, -0.5f);
  return vxe_fmaf(s, p, 1.0f);
}

/* sin / cos of |x| > 65536 (and NaN / inf): binary64 reduction. */
VXE_HD float vxe_sincos_wide(double x, int cosine) {
  if (x != x || x - x != 0.0) return (float)(x - x); /* NaN for NaN / inf */
  if (x > 1e18 || x < -1e18) return cosine ? 1.0f : 0.0f; /* beyond the reduction */
  int q;
  const double r = vxe_reduce_pio2(x, &q);
  q = (q + cosine) & 3;
  double v;
  if (q == 0) v = vxe_sin_poly(r);
  else if (q == 1) v = vxe_cos_poly(r);
  else if (q == 2) v = -vxe_sin_poly(r);
  else v = -vxe_cos_poly(r);
  return (float)v;
}

VXE_HD_CALL float vxe_sinf(float x) {
  if (!(x >= -65536.0f && x <= 65536.0f)) return vxe_sincos_wide((double)x, 0);
  int q;
  const float r = vxe_reduce_pio2f(x, &q);
  if (q == 0) return vxe_sin_polyf(r);
  if (q == 1) return vxe_cos_polyf(r);
  if (q == 2) return -vxe_sin_polyf(r);
  return -vxe_cos_polyf(r);
}

VXE_HD_CALL float vxe_cosf(float x) {
  if (!(x >= -65536.0f && x <= 65536.0f)) return vxe_sincos_wide((double)x, 1);
  int q;
  const float r = vxe_reduce_pio2f(x, &q);
  if (q == 0) return vxe_cos_polyf(r);
  if (q == 1) return -vxe_sin_polyf(r);
  if (q == 2) return -vxe_cos_polyf(r);
  return vxe_sin_polyf(r);
}

/* e^x in binary32: x = k ln 2 + r (fused Cody-Waite, ln 2 split at 16
 * significant bits), e^r = 1 + r q(r) with q the Taylor series of
 * (e^r - 1) / r to degree 7, then the exact scale by 2^k. */
VXE_HD_CALL float vxe_expf(float x) {
  if (x != x) return x;
  if (x > 88.72283935546875f) return vxe_u2f(0x7F800000u);
  if (x < -103.97208404541015625f) return 0.0f;
  const float kf = vxe_rintf(x * 1.4426950216293335f);
  float r = vxe_fmaf(-kf, 0.693145751953125f, x);
  r = vxe_fmaf(-kf, 1.428606765330187e-06f, r);
  float q = 1.0f / 40320.0f;
  q = vxe_fmaf(q, r, 1.0f / 5040.0f);
  q = vxe_fmaf(q, r, 1.0f / 720.0f);
  q = vxe_fmaf(q, r, 1.0f / 120.0f);
  q = vxe_fmaf(q, r, 1.0f / 24.0f);
  q = vxe_fmaf(q, r, 1.0f / 6.0f);
  q = vxe_fmaf(q, r, 0.5f);
  q = vxe_fmaf(q, r, 1.0f);
  const float e = vxe_fmaf(r, q, 1.0f);
  const int k = (int)kf;
  if (k > 127) return (e * 2.0f) * vxe_pow2if(k - 1);
  if (k < -125) return (e * vxe_pow2if(k + 64)) * vxe_pow2if(-64);
  return e * vxe_pow2if(k);
}

/* pow for the non-negative bases the passes use: pow(0, y>0) = 0,
 * pow(x, 0) = 1, negative bases give NaN (WGSL leaves them undefined).
 * Binary32 throughout: log x as an unevaluated sum hi + lo (x = 2^e m, m in
 * [sqrt(1/2), sqrt(2)), log m = 2 atanh(s) with s = (m-1)/(m+1) split hi + lo
 * by a fused residual, the larger parts summed by two-sums), y log x as
 * hi + lo (fused products), then e^t as in vxe_expf with the low part added
 * to the reduced argument. */
VXE_HD_CALL float vxe_powf(float x, float y) {
  if (y == 0.0f) return 1.0f;
  if (x == 0.0f) return y > 0.0f ? 0.0f : vxe_u2f(0x7F800000u);
  if (x == 1.0f) return 1.0f;
  if (!(x > 0.0f)) return vxe_u2f(0x7FC00000u);
  if (x == vxe_u2f(0x7F800000u)) return y > 0.0f ? x : 0.0f;
  if (y != y) return y;
  uint32_t u = vxe_f2u(x);
  int e = (int)((u >> 23) & 0xFFu);
  if (e == 0) {
    u = vxe_f2u(x * 16777216.0f);
    e = (int)((u >> 23) & 0xFFu) - 24;
  }
  e -= 127;
  float m = vxe_u2f((u & 0x007FFFFFu) | 0x3F800000u);
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  const float num = m - 1.0f;                     /* exact */
  const float den = m + 1.0f;                     /* den + dlo = m + 1 exactly (two-sum) */
  const float bb = den - m;
  const float dlo = (m - (den - bb)) + (1.0f - bb);
  const float rd = vxe_rcpf(den);
  const float s_hi = num * rd;
  const float res = vxe_fmaf(-s_hi, dlo, vxe_fmaf(-s_hi, den, num));
  const float s_lo = res * rd;
  const float s2 = s_hi * s_hi;
  float q = 2.0f / 13.0f;
  q = vxe_fmaf(q, s2, 2.0f / 11.0f);
  q = vxe_fmaf(q, s2, 2.0f / 9.0f);
  q = vxe_fmaf(q, s2, 2.0f / 7.0f);
  q = vxe_fmaf(q, s2, 2.0f / 5.0f);
  q = vxe_fmaf(q, s2, 2.0f / 3.0f);
  const float tail = (s2 * s_hi) * q;             /* log m - 2 s */
  const float ef = (float)e;
  const float a = ef * 0.693145751953125f;        /* exact: 16-bit constant, |e| < 2^8 */
  const float b = 2.0f * s_hi;
  const float l_hi = a + b;                        /* two-sum of a + b */
  const float bv = l_hi - a;
  const float l_err = (a - (l_hi - bv)) + (b - bv);
  const float l_lo = l_err + (2.0f * s_lo + tail) + ef * 1.428606765330187e-06f;
  const float t_hi = y * l_hi;
  const float t_lo = vxe_fmaf(y, l_lo, vxe_fmaf(y, l_hi, -t_hi));
  if (t_hi > 88.72283935546875f) return vxe_u2f(0x7F800000u);
  if (t_hi < -103.97208404541015625f) return 0.0f;
  const float kf = vxe_rintf(t_hi * 1.4426950216293335f);
  float r = vxe_fmaf(-kf, 0.693145751953125f, t_hi);  /* exact */
  r = vxe_fmaf(-kf, 1.428606765330187e-06f, r) + t_lo;
  float p = 1.0f / 40320.0f;
  p = vxe_fmaf(p, r, 1.0f / 5040.0f);
  p = vxe_fmaf(p, r, 1.0f / 720.0f);
  p = vxe_fmaf(p, r, 1.0f / 120.0f);
  p = vxe_fmaf(p, r, 1.0f / 24.0f);
  p = vxe_fmaf(p, r, 1.0f / 6.0f);
  p = vxe_fmaf(p, r, 0.5f);
  p = vxe_fmaf(p, r, 1.0f);
  const float ex = vxe_fmaf(r, p, 1.0f);
  const int k = (int)kf;
  if (k > 127) return (ex * 2.0f) * vxe_pow2if(k - 1);
  if (k < -125) return (ex * vxe_pow2if(k + 64)) * vxe_pow2if(-64);
  return ex * vxe_pow2if(k);
}

#endif /* VXE_DETMATH_H */
