/*
 * cplx.h -- double-complex arithmetic with a fixed evaluation order, usable
 * from host C/C++ and CUDA device code.
 *
 * The opacity kernels must round exactly like the CPU oracle, so complex
 * multiply and divide are written out here instead of relying on C99
 * _Complex or thrust::complex (whose division algorithms differ between
 * compilers).  Division uses Smith's algorithm (R. L. Smith, CACM 5, 435,
 * 1962), the method Fortran compilers use for COMPLEX division.
 */
#ifndef MCMAX_CPLX_H
#define MCMAX_CPLX_H

#include <math.h>

#if defined(__CUDACC__)
#define CX_FN static __host__ __device__ __forceinline__
#else
#define CX_FN static inline
#endif

typedef struct {
  double re, im;
} cx;

CX_FN cx cx_make(double re, double im) {
  cx z;
  z.re = re;
  z.im = im;
  return z;
}
CX_FN cx cx_add(cx a, cx b) { return cx_make(a.re + b.re, a.im + b.im); }
CX_FN cx cx_sub(cx a, cx b) { return cx_make(a.re - b.re, a.im - b.im); }
CX_FN cx cx_neg(cx a) { return cx_make(-a.re, -a.im); }
CX_FN cx cx_conj(cx a) { return cx_make(a.re, -a.im); }
CX_FN cx cx_mul(cx a, cx b) {
  double p = a.re * b.re;
  double q = a.im * b.im;
  double r = a.re * b.im;
  double s = a.im * b.re;
  return cx_make(p - q, r + s);
}
/* real scalar times complex */
CX_FN cx cx_scale(double s, cx a) { return cx_make(s * a.re, s * a.im); }
CX_FN cx cx_div(cx a, cx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re;
    double d = b.re + b.im * r;
    return cx_make((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  } else {
    double r = b.re / b.im;
    double d = b.im + b.re * r;
    return cx_make((a.re * r + a.im) / d, (a.im * r - a.re) / d);
  }
}
/* real scalar divided by complex */
CX_FN cx cx_rdiv(double s, cx b) { return cx_div(cx_make(s, 0.0), b); }
/* |z|^2 */
CX_FN double cx_abs2(cx a) { return a.re * a.re + a.im * a.im; }
/* |z| (plain sqrt of the sum of squares; arguments here never overflow) */
CX_FN double cx_abs(cx a) { return sqrt(a.re * a.re + a.im * a.im); }
/* principal square root, Re(result) >= 0 */
CX_FN cx cx_sqrt(cx z) {
  double a = cx_abs(z);
  if (a == 0.0) return cx_make(0.0, 0.0);
  if (z.re >= 0.0) {
    double t = sqrt(0.5 * (a + z.re));
    return cx_make(t, z.im / (2.0 * t));
  } else {
    double t = sqrt(0.5 * (a - z.re));
    return cx_make(fabs(z.im) / (2.0 * t), z.im >= 0.0 ? t : -t);
  }
}

#endif /* MCMAX_CPLX_H */
