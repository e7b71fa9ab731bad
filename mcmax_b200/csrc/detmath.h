/*
 * detmath.h -- deterministic elementary functions for host (C/C++) and
 * device (CUDA) code.
 *
 * Why this exists: the FP64 opacity path must produce bit-identical tables on
 * the GPU and in the CPU oracle.  glibc's libm and CUDA's libdevice round
 * sin/cos/exp/log differently in the last bit, so every transcendental that
 * feeds an FP64 result on the bit-exact path goes through these functions
 * instead.  They use only IEEE-754 operations that are correctly rounded on
 * both sides (add, mul, div, sqrt, fma, rint), so the same source gives the
 * same bits on x86-64 (SSE2, -ffp-contract=off) and on sm_100a (--fmad=false).
 *
 * Methods (all standard numerical analysis, constants derived for this file
 * with 300-bit arithmetic):
 *   exp: Cody-Waite reduction x = k ln2 + r with ln2 split into a 32-bit head
 *        and a tail, Taylor series of e^r to degree 13 (|r| <= ln2/2,
 *        truncation < 5e-18), exact scaling by 2^k.
 *   log: x = 2^e m, m in [sqrt(2)/2, sqrt(2)), log m = 2 atanh(s),
 *        s = (m-1)/(m+1), odd series in s to s^23 (|s| <= 0.1716).
 *   sin/cos: reduction by pi/2 split into three 33/33/53-bit parts (exact
 *        products for |k| < 2^20, i.e. |x| < 1.6e6), Taylor series on
 *        |r| <= pi/4.
 * Accuracy against glibc is checked in tests (a few ulp).  These functions
 * are NOT faster than the hardware/libm ones; the mixed-precision transport
 * path does not use them.
 */
#ifndef MCMAX_DETMATH_H
#define MCMAX_DETMATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define DM_FN static __host__ __device__ __forceinline__
#else
#define DM_FN static inline
#endif

DM_FN double dm_bits2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, sizeof d);
  return d;
#endif
}

DM_FN uint64_t dm_d2bits(double d) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  memcpy(&u, &d, sizeof u);
  return u;
#endif
}

/* 2^k as a double for k in [-1022, 1023] */
DM_FN double dm_pow2i(int k) { return dm_bits2d((uint64_t)(k + 1023) << 52); }

#define DM_LN2_HI 0x1.62e42fee00000p-1
#define DM_LN2_LO 0x1.a39ef35793c76p-33
#define DM_INV_LN2 1.4426950408889634
#define DM_PIO2_1 0x1.921fb54400000p+0
#define DM_PIO2_2 0x1.0b4611a600000p-34
#define DM_PIO2_3 0x1.3198a2e037073p-69
#define DM_TWO_OVER_PI 0.6366197723675814

/* e^x */
DM_FN double dm_exp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return HUGE_VAL;
  if (x < -745.2) return 0.0;
  double k = rint(x * DM_INV_LN2);
  double r = fma(-k, DM_LN2_HI, x);
  r = fma(-k, DM_LN2_LO, r);
  /* Taylor coefficients 1/n!, n = 13 .. 2 */
  double p = 0x1.6124613a86d09p-33;  /* 1/13! */
  p = fma(p, r, 0x1.1eed8eff8d898p-29);  /* 1/12! */
  p = fma(p, r, 0x1.ae64567f544e4p-26);  /* 1/11! */
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);  /* 1/10! */
  p = fma(p, r, 0x1.71de3a556c734p-19);  /* 1/9! */
  p = fma(p, r, 0x1.a01a01a01a01ap-16);  /* 1/8! */
  p = fma(p, r, 0x1.a01a01a01a01ap-13);  /* 1/7! */
  p = fma(p, r, 0x1.6c16c16c16c17p-10);  /* 1/6! */
  p = fma(p, r, 0x1.1111111111111p-7);   /* 1/5! */
  p = fma(p, r, 0x1.5555555555555p-5);   /* 1/4! */
  p = fma(p, r, 0x1.5555555555555p-3);   /* 1/3! */
  p = fma(p, r, 0.5);                       /* 1/2! */
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  int ki = (int)k;
  if (ki > 1023) return (p * dm_pow2i(1023)) * 2.0;
  if (ki < -1022) return (p * dm_pow2i(ki + 600)) * dm_pow2i(-600);
  return p * dm_pow2i(ki);
}

/* natural logarithm */
DM_FN double dm_log(double x) {
  if (x != x) return x;
  if (x < 0.0) return (x - x) / (x - x); /* NaN */
  if (x == 0.0) return -HUGE_VAL;
  if (x == HUGE_VAL) return x;
  int e = 0;
  if (x < 0x1p-1022) { x *= 0x1p54; e = -54; }
  uint64_t u = dm_d2bits(x);
  e += (int)((u >> 52) & 0x7ff) - 1023;
  double m = dm_bits2d((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > 1.4142135623730951) { m *= 0.5; e += 1; }
  double f = m - 1.0;
  double s = f / (2.0 + f);
  double t = s * s;
  /* sum_{n=0}^{11} t^n/(2n+1) */
  double p = 0x1.642c8590b2164p-5; /* 1/23 */
  p = fma(p, t, 0x1.8618618618618p-5); /* 1/21 */
  p = fma(p, t, 0x1.af286bca1af28p-5); /* 1/19 */
  p = fma(p, t, 0x1.e1e1e1e1e1e1ep-5); /* 1/17 */
  p = fma(p, t, 0x1.1111111111111p-4); /* 1/15 */
  p = fma(p, t, 0x1.3b13b13b13b14p-4); /* 1/13 */
  p = fma(p, t, 0x1.745d1745d1746p-4); /* 1/11 */
  p = fma(p, t, 0x1.c71c71c71c71cp-4); /* 1/9 */
  p = fma(p, t, 0x1.2492492492492p-3); /* 1/7 */
  p = fma(p, t, 0x1.999999999999ap-3); /* 1/5 */
  p = fma(p, t, 0x1.5555555555555p-2); /* 1/3 */
  /* log m = 2s + 2 s t p  (the leading term kept separate for accuracy) */
  double lm = fma(2.0 * s * t, p, 2.0 * s);
  double de = (double)e;
  return fma(de, DM_LN2_HI, fma(de, DM_LN2_LO, lm));
}

/* polynomials on the reduced interval |r| <= pi/4 */
DM_FN double dm_sin_poly(double r) {
  double z = r * r;
  double p = -0x1.71b8ef6dcf572p-66; /* -1/21! */
  p = fma(p, z, 0x1.2f49b46814157p-57); /* 1/19! */
  p = fma(p, z, -0x1.952c77030ad4ap-49); /* -1/17! */
  p = fma(p, z, 0x1.ae7f3e733b81fp-41); /* 1/15! */
  p = fma(p, z, -0x1.6124613a86d09p-33); /* -1/13! */
  p = fma(p, z, 0x1.ae64567f544e4p-26); /* 1/11! */
  p = fma(p, z, -0x1.71de3a556c734p-19); /* -1/9! */
  p = fma(p, z, 0x1.a01a01a01a01ap-13); /* 1/7! */
  p = fma(p, z, -0x1.1111111111111p-7); /* -1/5! */
  p = fma(p, z, 0x1.5555555555555p-3); /* 1/3! */
  /* sin r = r - r z (1/6 - z/120 + ...) */
  return fma(-(r * z), p, r);
}

DM_FN double dm_cos_poly(double r) {
  double z = r * r;
  double p = 0x1.e542ba4020225p-62;  /* 1/20! */
  p = fma(p, z, -0x1.6827863b97d97p-53); /* -1/18! */
  p = fma(p, z, 0x1.ae7f3e733b81fp-45); /* 1/16! */
  p = fma(p, z, -0x1.93974a8c07c9dp-37); /* -1/14! */
  p = fma(p, z, 0x1.1eed8eff8d898p-29); /* 1/12! */
  p = fma(p, z, -0x1.27e4fb7789f5cp-22); /* -1/10! */
  p = fma(p, z, 0x1.a01a01a01a01ap-16); /* 1/8! */
  p = fma(p, z, -0x1.6c16c16c16c17p-10); /* -1/6! */
  p = fma(p, z, 0x1.5555555555555p-5); /* 1/4! */
  /* cos r = 1 - z/2 + z^2 (1/24 - ...) */
  double hz = 0.5 * z;
  double w = 1.0 - hz;
  return w + (((1.0 - w) - hz) + (z * z) * p);
}

DM_FN void dm_reduce_pio2(double x, double *r, int *q) {
  double k = rint(x * DM_TWO_OVER_PI);
  double t = fma(-k, DM_PIO2_1, x);
  t = fma(-k, DM_PIO2_2, t);
  t = fma(-k, DM_PIO2_3, t);
  *r = t;
  long long ki = (long long)k;
  *q = (int)(ki & 3);
}

DM_FN double dm_sin(double x) {
  if (x != x || x == HUGE_VAL || x == -HUGE_VAL) return (x - x) / (x - x);
  double r;
  int q;
  dm_reduce_pio2(x, &r, &q);
  switch (q) {
    case 0: return dm_sin_poly(r);
    case 1: return dm_cos_poly(r);
    case 2: return -dm_sin_poly(r);
    default: return -dm_cos_poly(r);
  }
}

DM_FN double dm_cos(double x) {
  if (x != x || x == HUGE_VAL || x == -HUGE_VAL) return (x - x) / (x - x);
  double r;
  int q;
  dm_reduce_pio2(x, &r, &q);
  switch (q) {
    case 0: return dm_cos_poly(r);
    case 1: return -dm_sin_poly(r);
    case 2: return -dm_cos_poly(r);
    default: return dm_sin_poly(r);
  }
}

/* x^(1/3) for x > 0 (used only where the result is truncated to an integer
 * term count, so a few ulp do not matter; it must only be deterministic) */
DM_FN double dm_cbrt_pos(double x) { return dm_exp(dm_log(x) * (1.0 / 3.0)); }

#endif /* MCMAX_DETMATH_H */
