/*
 * dhs_core.cuh -- per-sample light-scattering cores of the opacity stage,
 * written once for the GPU (one warp per sample, NL = 32 lanes) and
 * compilable for the host (NL = 1) so the same source can be replayed on the
 * CPU against the oracle.
 *
 *   dhs_sample  coated sphere of Toon & Ackerman (1981), Appl. Opt. 20, 3657,
 *               in the formulation of ComputePart.f:1256-1711 (DMiLay):
 *               down-recurrences for A_n and W_n(z) (4 independent chains,
 *               run by 4 lanes), then the upward Mie sum; the scalar chain
 *               (coefficients a_n, b_n) is evaluated redundantly by every
 *               lane, the 90 scattering-angle sums are split across lanes.
 *   mie_sample  homogeneous sphere, de Rooij & van der Stap (1984) as in
 *               ComputePart.f:1883-3213 (MeerhoffMie/scatmat/fichid/anbn/
 *               pitau): recurrences by three lanes, a_n, b_n in parallel over
 *               n, the angle sums in parallel over angles with pi_n/tau_n
 *               generated on the fly.
 *
 * Every floating-point operation keeps the order of the oracle (oracle/) so
 * that FP64 results agree bit for bit; this translation unit is compiled with
 * --fmad=false and all transcendentals come from detmath.h.
 */
#ifndef MCMAX_DHS_CORE_CUH
#define MCMAX_DHS_CORE_CUH

#include "cplx.h"
#include "detmath.h"

#if defined(__CUDACC__)
#define DH_FN __host__ __device__ __forceinline__
#else
#define DH_FN static inline
#endif

#define DHS_PI 3.14159265358979323846
#define DHS_LL 200000
#define DHS_NUMANG 90

/* synchronise the lanes that cooperate on one sample */
template <int NL>
DH_FN void lanes_sync() {
#if defined(__CUDA_ARCH__)
  if (NL > 1) __syncwarp();
#endif
}

/* broadcast an int from lane 0 */
template <int NL>
DH_FN int lanes_bcast_int(int v) {
#if defined(__CUDA_ARCH__)
  if (NL > 1) return __shfl_sync(0xffffffffu, v, 0);
#endif
  return v;
}

/* NMX1 of DMiLay for a shell of size parameter xshell and index |m| */
DH_FN int dhs_nmx1(double rshell, double wvno, double m_re, double m_im) {
  double xshell = rshell * wvno;
  double t1 = xshell * cx_abs(cx_make(m_re, m_im));
  double f = 1.1 * t1;
  if (!(f < 2.0e9)) return 2000000000;
  int n = (int)f;
  return n <= 150 ? 150 : n;
}

/* One coated-sphere evaluation (vacuum core, shell index m = m_re - i m_im
 * with m_im >= 0 passed as the reference passes it: RINDSH = (e1, -e2)).
 * scratch: 4*cap complex values, cap >= NMX1+2.
 * Outputs (lane-distributed): F11/F12/F33/F34 of the 180 bins as formed in
 * ComputePart.f:391-404 (before the forward-peak renormalisation), and
 * cemie/csmie.  Returns 0, or 1 for the reference's Err = 1. */
template <int NL, int APL>
DH_FN int dhs_sample(double rcore, double rshell, double wvno, double sh_re, double sh_im,
                     const double *mu_tab, cx *scratch, int cap, int lane, double *F11,
                     double *F12, double *F33, double *F34, double *cemie_out,
                     double *csmie_out) {
  const cx CI = cx_make(0.0, 1.0);
  const cx rindsh = cx_make(sh_re, sh_im);
  const cx rindco = cx_make(1.0, 0.0);
  const double xshell = rshell * wvno;
  const double xcore = rcore * wvno;
  const double t1a = xshell * cx_abs(rindsh);
  const double fn1 = 1.1 * t1a;
  if (!(fn1 < 2.0e9)) return 1;
  int nmx1 = (int)fn1;
  int nmx2 = (int)t1a;
  if (nmx1 <= 150) {
    nmx1 = 150;
    nmx2 = 135;
  }
  if (wvno <= 0.0 || rshell <= 0.0 || rcore <= 0.0 || rcore > rshell) return 1;
  if (rindsh.re <= 0.0 || rindsh.im > 0.0) return 1;
  if (nmx1 + 1 > DHS_LL || nmx1 + 2 > cap) return 1;

  const cx k1 = cx_scale(wvno, rindco);
  const cx k2 = cx_scale(wvno, rindsh);
  const cx k3 = cx_make(wvno, 0.0);
  cx z1 = cx_scale(xshell, rindsh);
  cx z2 = cx_make(xshell, 0.0);
  cx z3 = cx_scale(xcore, rindco);
  cx z4 = cx_scale(xcore, rindsh);
  const double x1 = z1.re, y1 = z1.im, x4 = z4.re, y4 = z4.im;
  const double rx = 1.0 / xshell;

  cx *acap = scratch;
  cx *w1 = scratch + cap;
  cx *w2 = scratch + 2 * cap;
  cx *w3 = scratch + 3 * cap;

  /* four independent down-recurrences, one per lane (ComputePart.f:1439-1454) */
  for (int ch = lane; ch < 4; ch += NL) {
    cx *dst = scratch + (size_t)ch * cap;
    dst[nmx1 + 1] = cx_make(0.0, 0.0);
    if (ch == 0) {
      cx rrfx = cx_rdiv(1.0, cx_scale(xshell, rindsh));
      for (int nn = nmx1; nn >= 1; --nn) {
        cx a = cx_scale((double)(nn + 1), rrfx);
        dst[nn] = cx_sub(a, cx_rdiv(1.0, cx_add(a, dst[nn + 1])));
      }
    } else {
      cx zz = ch == 1 ? z2 : (ch == 2 ? z3 : z4);
      for (int nn = nmx1; nn >= 1; --nn) {
        cx b = cx_rdiv((double)(nn + 1), zz);
        dst[nn] = cx_sub(b, cx_rdiv(1.0, cx_add(b, dst[nn + 1])));
      }
    }
  }
  lanes_sync<NL>();

  /* lane-private angle state */
  double mu[APL], si2[APL], pi0[APL], pi1[APL], pi2[APL], ta0[APL], ta1[APL], ta2[APL];
  cx s1a[APL], s1b[APL], s2a[APL], s2b[APL];
#pragma unroll
  for (int a = 0; a < APL; ++a) {
    int j = lane + a * NL;
    double m = j < DHS_NUMANG ? mu_tab[j] : 0.0;
    mu[a] = m;
    si2[a] = 1.0 - m * m;
    pi0[a] = 0.0;
    pi1[a] = 1.0;
    ta0[a] = 0.0;
    ta1[a] = m;
  }

  double t1 = dm_cos(xshell), t2 = dm_sin(xshell);
  cx wm1 = cx_make(t1, -t2);
  cx wfn1 = cx_make(t2, t1);
  cx wfn2 = cx_sub(cx_scale(rx, wfn1), wm1);
  double ta3 = wfn2.re;

  int n = 1;
  const double sinx1 = dm_sin(x1), sinx4 = dm_sin(x4), cosx1 = dm_cos(x1), cosx4 = dm_cos(x4);
  const double ey1 = dm_exp(y1);
  const double e2y1 = ey1 * ey1;
  const double ey4 = dm_exp(y4);
  const double ey1my4 = dm_exp(y1 - y4);
  const double ey1py4 = ey1 * ey4;
  const double aa = sinx4 * (ey1py4 + ey1my4);
  const double bb = cosx4 * (ey1py4 - ey1my4);
  const double cc = sinx1 * (e2y1 + 1.0);
  const double dd = cosx1 * (e2y1 - 1.0);
  const double denom = 1.0 + e2y1 * ((4.0 * (sinx1 * sinx1) - 2.0) + e2y1);
  cx dummy = cx_make((aa * cc + bb * dd) / denom, (bb * cc - aa * dd) / denom);
  cx nz1 = cx_rdiv((double)n, z1);
  cx nz4 = cx_rdiv((double)n, z4);
  cx a_n = acap[n], w1n = w1[n], w2n = w2[n], w3n = w3[n];
  dummy = cx_div(cx_mul(dummy, cx_add(a_n, nz1)), cx_add(w3n, nz4));
  cx dumsq = cx_mul(dummy, dummy);
  cx p24h24 = cx_scale(ey4 * ey4, cx_make(sinx4 * sinx4 - 0.5, cosx4 * sinx4));
  p24h24 = cx_make(0.5 + p24h24.re, p24h24.im);
  cx p24h21 = cx_add(
      cx_scale(ey1py4, cx_scale(0.5, cx_make(sinx1 * sinx4 - cosx1 * cosx4,
                                             sinx1 * cosx4 + cosx1 * sinx4))),
      cx_scale(ey1my4, cx_scale(0.5, cx_make(sinx1 * sinx4 + cosx1 * cosx4,
                                             -(sinx1 * cosx4) + cosx1 * sinx4))));
  const cx one = cx_make(1.0, 0.0);
  cx dh1 = cx_sub(cx_div(z1, cx_add(one, cx_mul(CI, z1))), cx_rdiv(1.0, z1));
  cx dh2 = cx_sub(cx_div(z2, cx_add(one, cx_mul(CI, z2))), cx_rdiv(1.0, z2));
  cx dh4 = cx_sub(cx_div(z4, cx_add(one, cx_mul(CI, z4))), cx_rdiv(1.0, z4));
  p24h24 = cx_div(p24h24, cx_mul(cx_add(dh4, nz4), cx_add(w3n, nz4)));
  p24h21 = cx_div(p24h21, cx_mul(cx_add(dh1, nz1), cx_add(w3n, nz4)));

  cx u1 = cx_sub(cx_mul(k3, a_n), cx_mul(k2, w1n));
  cx u2 = cx_sub(cx_mul(k3, a_n), cx_mul(k2, dh2));
  cx u3 = cx_sub(cx_mul(k2, a_n), cx_mul(k3, w1n));
  cx u4 = cx_sub(cx_mul(k2, a_n), cx_mul(k3, dh2));
  cx u5 = cx_sub(cx_mul(k1, w3n), cx_mul(k2, w2n));
  cx u6 = cx_sub(cx_mul(k2, w3n), cx_mul(k1, w2n));
  cx u7 = cx_neg(cx_mul(CI, cx_sub(cx_mul(dummy, p24h21), p24h24)));
  cx u8 = cx_rdiv(ta3, wfn2);
  cx d35 = cx_mul(cx_mul(dumsq, k3), u5);
  cx d26 = cx_mul(cx_mul(dumsq, k2), u6);
  cx acoe = cx_div(cx_mul(u8, cx_sub(cx_add(cx_mul(cx_mul(u1, u5), u7), cx_mul(k1, u1)), d35)),
                   cx_sub(cx_add(cx_mul(cx_mul(u2, u5), u7), cx_mul(k1, u2)), d35));
  cx bcoe = cx_div(cx_mul(u8, cx_sub(cx_add(cx_mul(cx_mul(u3, u6), u7), cx_mul(k2, u3)), d26)),
                   cx_sub(cx_add(cx_mul(cx_mul(u4, u6), u7), cx_mul(k2, u4)), d26));
  double are = acoe.re, aim = acoe.im, bre = bcoe.re, bim = bcoe.im;
  double dqext = 3.0 * (are + bre);
  double dqsca = 3.0 * (((are * are + aim * aim) + bre * bre) + bim * bim);
  cx ac = cx_scale(1.5, acoe);
  cx bc = cx_scale(1.5, bcoe);
#pragma unroll
  for (int a = 0; a < APL; ++a) {
    cx ap = cx_scale(pi1[a], ac), bt = cx_scale(ta1[a], bc);
    cx bp = cx_scale(pi1[a], bc), at = cx_scale(ta1[a], ac);
    s1a[a] = cx_add(ap, bt);
    s1b[a] = cx_sub(ap, bt);
    s2a[a] = cx_add(bp, at);
    s2b[a] = cx_sub(bp, at);
  }

  int err = 0;
  n = 2;
  for (;;) {
    const double tn1 = (double)(2 * n - 1);
    const double tn2 = (double)(n - 1);
    const double dn = (double)n;
#pragma unroll
    for (int a = 0; a < APL; ++a) {
      pi2[a] = ((tn1 * pi1[a]) * mu[a] - dn * pi0[a]) / tn2;
      ta2[a] = (mu[a] * (pi2[a] - pi0[a]) - (tn1 * si2[a]) * pi1[a]) + ta0[a];
    }
    wm1 = wfn1;
    wfn1 = wfn2;
    wfn2 = cx_sub(cx_scale(tn1 * rx, wfn1), wm1);
    ta3 = wfn2.re;

    a_n = acap[n];
    w1n = w1[n];
    w2n = w2[n];
    w3n = w3[n];
    nz1 = cx_rdiv(dn, z1);
    cx nz2 = cx_rdiv(dn, z2);
    nz4 = cx_rdiv(dn, z4);
    dh1 = cx_add(cx_neg(nz1), cx_rdiv(1.0, cx_sub(nz1, dh1)));
    dh2 = cx_add(cx_neg(nz2), cx_rdiv(1.0, cx_sub(nz2, dh2)));
    dh4 = cx_add(cx_neg(nz4), cx_rdiv(1.0, cx_sub(nz4, dh4)));
    cx w3nz4 = cx_add(w3n, nz4);
    p24h24 = cx_div(p24h24, cx_mul(cx_add(dh4, nz4), w3nz4));
    p24h21 = cx_div(p24h21, cx_mul(cx_add(dh1, nz1), w3nz4));
    dummy = cx_div(cx_mul(dummy, cx_add(a_n, nz1)), w3nz4);
    dumsq = cx_mul(dummy, dummy);

    u1 = cx_sub(cx_mul(k3, a_n), cx_mul(k2, w1n));
    u2 = cx_sub(cx_mul(k3, a_n), cx_mul(k2, dh2));
    u3 = cx_sub(cx_mul(k2, a_n), cx_mul(k3, w1n));
    u4 = cx_sub(cx_mul(k2, a_n), cx_mul(k3, dh2));
    u5 = cx_sub(cx_mul(k1, w3n), cx_mul(k2, w2n));
    u6 = cx_sub(cx_mul(k2, w3n), cx_mul(k1, w2n));
    u7 = cx_neg(cx_mul(CI, cx_sub(cx_mul(dummy, p24h21), p24h24)));
    u8 = cx_rdiv(ta3, wfn2);
    d35 = cx_mul(cx_mul(dumsq, k3), u5);
    d26 = cx_mul(cx_mul(dumsq, k2), u6);
    acoe = cx_div(cx_mul(u8, cx_sub(cx_add(cx_mul(cx_mul(u1, u5), u7), cx_mul(k1, u1)), d35)),
                  cx_sub(cx_add(cx_mul(cx_mul(u2, u5), u7), cx_mul(k1, u2)), d35));
    bcoe = cx_div(cx_mul(u8, cx_sub(cx_add(cx_mul(cx_mul(u3, u6), u7), cx_mul(k2, u3)), d26)),
                  cx_sub(cx_add(cx_mul(cx_mul(u4, u6), u7), cx_mul(k2, u4)), d26));
    are = acoe.re;
    aim = acoe.im;
    bre = bcoe.re;
    bim = bcoe.im;

    const double t3 = (double)(2 * n + 1);
    dqext = dqext + t3 * (are + bre);
    const double t4 = ((are * are + aim * aim) + bre * bre) + bim * bim;
    dqsca = dqsca + t3 * t4;
    const double tt = t3 / (double)(n * (n + 1));
    ac = cx_scale(tt, acoe);
    bc = cx_scale(tt, bcoe);
    const bool even = (n & 1) == 0;
#pragma unroll
    for (int a = 0; a < APL; ++a) {
      cx ap = cx_scale(pi2[a], ac), bt = cx_scale(ta2[a], bc);
      cx bp = cx_scale(pi2[a], bc), at = cx_scale(ta2[a], ac);
      s1a[a] = cx_add(cx_add(s1a[a], ap), bt);
      s2a[a] = cx_add(cx_add(s2a[a], bp), at);
      if (even) {
        s1b[a] = cx_add(cx_sub(s1b[a], ap), bt);
        s2b[a] = cx_add(cx_sub(s2b[a], bp), at);
      } else {
        s1b[a] = cx_sub(cx_add(s1b[a], ap), bt);
        s2b[a] = cx_sub(cx_add(s2b[a], bp), at);
      }
    }
    if (t4 >= 1.0e-14) {
      n = n + 1;
      if (n > nmx2) {
        err = 1;
        break;
      }
#pragma unroll
      for (int a = 0; a < APL; ++a) {
        pi0[a] = pi1[a];
        pi1[a] = pi2[a];
        ta0[a] = ta1[a];
        ta1[a] = ta2[a];
      }
      continue;
    }
    break;
  }
  if (err) return 1;

  const double tq = 2.0 * (rx * rx);
  const double qext = tq * dqext;
  const double qsca = tq * dqsca;
  const double cemie = qext * DHS_PI * (rshell * rshell);
  const double csmie = qsca * DHS_PI * (rshell * rshell);
  const double wv2 = wvno * wvno;
#pragma unroll
  for (int a = 0; a < APL; ++a) {
    int j = lane + a * NL;
    if (j >= DHS_NUMANG) continue;
    for (int k = 0; k < 2; ++k) {
      cx sa = k == 0 ? s1a[a] : s1b[a];
      cx sb = k == 0 ? s2a[a] : s2b[a];
      double m1 = sa.re * sa.re + sa.im * sa.im;
      double m2 = sb.re * sb.re + sb.im * sb.im;
      double s21 = sa.re * sb.re + sa.im * sb.im;
      double d21 = sa.im * sb.re - sb.im * sa.re;
      int jj = k == 0 ? j : (2 * DHS_NUMANG - 1 - j);
      F11[jj] = (((m2 + m1) / csmie) / wv2) * 2.0 * DHS_PI;
      F12[jj] = (((m2 - m1) / csmie) / wv2) * 2.0 * DHS_PI;
      F33[jj] = ((s21 / csmie) / wv2) * 2.0 * DHS_PI;
      F34[jj] = ((-d21 / csmie) / wv2) * 2.0 * DHS_PI;
    }
  }
  *cemie_out = cemie;
  *csmie_out = csmie;
  return 0;
}

/* term counts of the homogeneous-sphere evaluation (scatmat :2968-2975) */
DH_FN void mie_counts(double rad, double lam, double e1, double e2, int *nmax, int *nfi, int *nD) {
  const double rtox = 2.0 * DHS_PI / lam;
  double x = rtox * rad;
  *nmax = (int)(x + 4.05 * dm_cbrt_pos(x) + 20.0);
  *nfi = *nmax + 60;
  double zabs = x * cx_abs(cx_make(e1, -e2));
  *nD = (int)(zabs + 4.05 * dm_cbrt_pos(zabs) + 70.0);
}

/* One homogeneous-sphere evaluation.  scratch: doubles, 8*cap entries with
 * cap >= max(nfi, nD) + 2.  Outputs F11..F34[180] (index 0 = most forward
 * bin) and csca/cext.  Returns 0, or 1 when the term counts do not fit. */
template <int NL, int APL>
DH_FN int mie_sample(double rad, double lam, double e1, double e2, double *scratch, int cap,
                     int lane, double *F11, double *F12, double *F33, double *F34,
                     double *csca_out, double *cext_out) {
  const double pie = DHS_PI;
  const double radfac = pie / 180.0;
  const double rtox = 2.0 * pie / lam;
  const double fakt = lam * lam / (2.0 * pie);
  const cx m = cx_make(e1, -e2);
  const double x = rtox * rad;
  int nmax, nfi, nD;
  mie_counts(rad, lam, e1, e2, &nmax, &nfi, &nD);
  if (nD < nmax || nmax < 2) return 1;
  if (nfi + 2 > cap || nD + 2 > cap) return 1;
  double *psi = scratch;
  double *chi = scratch + cap;
  cx *D = (cx *)(scratch + 2 * cap);
  cx *an = (cx *)(scratch + 4 * cap);
  cx *bn = (cx *)(scratch + 6 * cap);
  /* facf shares the chi slot beyond nmax? no: keep it in psi's tail-free
   * storage would alias; the 8*cap layout has no room, so facf is recomputed */

  const double perx = 1.0 / x;
  const double sinx = dm_sin(x), cosx = dm_cos(x);
  /* fichid, ComputePart.f:2506-2560: three independent recurrences */
  for (int t = lane; t < 3; t += NL) {
    if (t == 0) {
      psi[nfi] = 0.0;
      for (int k = nfi - 1; k >= 0; --k) psi[k] = 1.0 / ((double)(2 * k + 1) / x - psi[k + 1]);
      psi[0] = sinx;
      double psi1 = psi[0] * perx - cosx;
      if (fabs(psi1) > 1.0e-4) {
        psi[1] = psi1;
        for (int k = 2; k <= nmax; ++k) psi[k] = psi[k] * psi[k - 1];
      } else {
        for (int k = 1; k <= nmax; ++k) psi[k] = psi[k] * psi[k - 1];
      }
    } else if (t == 1) {
      cx zz = cx_scale(x, m);
      cx perz = cx_rdiv(1.0, zz);
      D[nD] = cx_make(0.0, 0.0);
      for (int k = nD - 1; k >= 1; --k) {
        cx zn1 = cx_scale((double)(k + 1), perz);
        D[k] = cx_sub(zn1, cx_rdiv(1.0, cx_add(D[k + 1], zn1)));
      }
    } else {
      chi[0] = cosx;
      chi[1] = chi[0] * perx + sinx;
      for (int k = 1; k <= nmax - 1; ++k) chi[k + 1] = ((double)(2 * k + 1) * chi[k]) * perx - chi[k - 1];
    }
  }
  lanes_sync<NL>();
  /* anbn, ComputePart.f:2211-2236, independent over n */
  {
    cx perm = cx_rdiv(1.0, m);
    for (int k = 1 + lane; k <= nmax; k += NL) {
      cx zn = cx_make(psi[k], chi[k]);
      cx znm1 = cx_make(psi[k - 1], chi[k - 1]);
      double xn = (double)k * perx;
      cx sv = cx_mul(D[k], perm);
      sv = cx_make(sv.re + xn, sv.im);
      cx num = cx_scale(psi[k], sv);
      num = cx_make(num.re - psi[k - 1], num.im);
      an[k] = cx_div(num, cx_sub(cx_mul(sv, zn), znm1));
      sv = cx_mul(m, D[k]);
      sv = cx_make(sv.re + xn, sv.im);
      num = cx_scale(psi[k], sv);
      num = cx_make(num.re - psi[k - 1], num.im);
      bn[k] = cx_div(num, cx_sub(cx_mul(sv, zn), znm1));
    }
  }
  lanes_sync<NL>();
  /* cross sections and truncation (scatmat :2995-3010), sequential order */
  double cextsum = 0.0, cscasum = 0.0;
  int nstop = nmax;
  for (int k = 1; k <= nmax; ++k) {
    cx aa = cx_mul(an[k], cx_conj(an[k]));
    cx bb = cx_mul(bn[k], cx_conj(bn[k]));
    double aux = (2.0 * (double)k + 1.0) * fabs(aa.re + bb.re);
    cscasum = cscasum + aux;
    cextsum = cextsum + (2.0 * (double)k + 1.0) * (an[k].re + bn[k].re);
    if (aux < 1.0e-8) {
      nstop = k;
      break;
    }
  }
  const int nfou = nstop;
  const double Csca0 = 1.0 * cscasum;
  const double Cext0 = 1.0 * cextsum;
  /* angle sums over j = 1..90 and their supplements */
#pragma unroll 1
  for (int a = 0; a < APL; ++a) {
    int j = 1 + lane + a * NL;
    if (j > DHS_NUMANG) continue;
    double th = 0.5 + (double)(180 - j) * 1.0; /* u(j) = cos((180.5-j) deg) */
    double uj = dm_cos(radfac * th);
    double p_prev = 1.0, p_cur = 3.0 * uj; /* pi(1), pi(2) */
    double delta = (3.0 * uj) * uj - 1.0;
    double t_prev = uj, t_cur = 2.0 * delta - 1.0;
    cx spf = cx_make(0, 0), smf = cx_make(0, 0), spb = cx_make(0, 0), smb = cx_make(0, 0);
    for (int k = 1; k <= nfou; ++k) {
      double pk, tk;
      if (k == 1) {
        pk = p_prev;
        tk = t_prev;
      } else {
        pk = p_cur;
        tk = t_cur;
        if (k >= 2 && k < nfou) {
          /* advance to k+1 (pitau, ComputePart.f:2733-2737) */
          double pn = ((double)(k + 1) / (double)k) * delta + uj * p_cur;
          delta = uj * pn - p_cur;
          double tn = (double)(k + 1) * delta - p_cur;
          p_prev = p_cur;
          p_cur = pn;
          t_prev = t_cur;
          t_cur = tn;
        }
      }
      double facf = (double)(2 * k + 1) / (double)(k * (k + 1));
      double facb = (k & 1) ? -facf : facf;
      cx apb = cx_add(an[k], bn[k]);
      cx amb = cx_sub(an[k], bn[k]);
      double ppt = pk + tk, pmt = pk - tk;
      spf = cx_add(spf, cx_scale(ppt, cx_scale(facf, apb)));
      smf = cx_add(smf, cx_scale(pmt, cx_scale(facf, amb)));
      spb = cx_add(spb, cx_scale(pmt, cx_scale(facb, apb)));
      smb = cx_add(smb, cx_scale(ppt, cx_scale(facb, amb)));
    }
    cx cspf = cx_conj(spf), csmf = cx_conj(smf), cspb = cx_conj(spb), csmb = cx_conj(smb);
    cx p, q;
    double f1, f2, f3, f4, b1, b2, b3, b4;
    p = cx_mul(spf, cspf); q = cx_mul(smf, csmf);
    f1 = 0.0 + 1.0 * (p.re + q.re);
    f3 = 0.0 + 1.0 * (p.re - q.re);
    p = cx_mul(smf, cspf); q = cx_mul(spf, csmf);
    f2 = 0.0 - 1.0 * (p.re + q.re);
    f4 = 0.0 + (0.0 * (p.re - q.re) - 1.0 * (p.im - q.im));
    p = cx_mul(spb, cspb); q = cx_mul(smb, csmb);
    b1 = 0.0 + 1.0 * (p.re + q.re);
    b3 = 0.0 + 1.0 * (p.re - q.re);
    p = cx_mul(smb, cspb); q = cx_mul(spb, csmb);
    b2 = 0.0 - 1.0 * (p.re + q.re);
    b4 = 0.0 + (0.0 * (p.re - q.re) - 1.0 * (p.im - q.im));
    const double d2 = 2.0 * Csca0;
    /* F(.,j) -> output bin 180-j (0-based), F(.,181-j) -> bin j-1 */
    F11[180 - j] = f1 / d2;
    F12[180 - j] = f2 / d2;
    F33[180 - j] = f3 / d2;
    F34[180 - j] = f4 / d2;
    F11[j - 1] = b1 / d2;
    F12[j - 1] = b2 / d2;
    F33[j - 1] = b3 / d2;
    F34[j - 1] = b4 / d2;
  }
  *csca_out = Csca0 * fakt;
  *cext_out = Cext0 * fakt;
  return 0;
}

#endif /* MCMAX_DHS_CORE_CUH */
