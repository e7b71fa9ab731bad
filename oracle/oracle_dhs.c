/*
 * oracle_dhs.c -- CPU restatement of MCMax's opacity stage (ComputePart.f),
 * test infrastructure only (see oracle.h for status and precision notes).
 *
 * Follows, in order:
 *   ComputePart  ComputePart.f:1-552   (size grid, filling-fraction grid,
 *                                       DHS / Mie selection, Mueller matrix,
 *                                       forward-peak renormalisation, mass
 *                                       opacities)
 *   Blender      ComputePart.f:1177-1212
 *   gauleg2      ComputePart.f:1219-1249
 *   DMiLay       ComputePart.f:1256-1711 (Toon & Ackerman 1981, Wiscombe's
 *                                         double-precision form)
 *   MeerhoffMie  ComputePart.f:1883-1927, mie :1932, scatmat :2882-3213,
 *                fichid :2506, anbn :2211, pitau :2719
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "../mcmax_b200/csrc/cplx.h"
#include "../mcmax_b200/csrc/detmath.h"

#define PI_D 3.14159265358979323846

/* ---------------------------------------------------------------- DMiLay */

#define DM_MXANG 200
#define DM_LL 200000

int orc_dmilay(double rcore, double rshell, double wvno, double shell_re, double shell_im,
               double core_re, double core_im, const double *mu, int numang, double *qext,
               double *qsca, double *qbs, double *gqsc, double *m1, double *m2, double *s21,
               double *d21) {
  const cx CI = cx_make(0.0, 1.0);
  cx rindsh = cx_make(shell_re, shell_im);
  cx rindco = cx_make(core_re, core_im);
  double xshell = rshell * wvno;
  double xcore = rcore * wvno;
  double t1 = xshell * cx_abs(rindsh);
  double fn1 = 1.1 * t1;
  if (!(fn1 < 2.0e9)) return 1;
  int nmx1 = (int)fn1;
  int nmx2 = (int)t1;
  if (nmx1 <= 150) {
    nmx1 = 150;
    nmx2 = 135;
  }
  /* gross input checks, ComputePart.f:1386-1420 */
  int inperr = 0;
  if (wvno <= 0.0) inperr = 1;
  if (rshell <= 0.0) inperr = 1;
  if (rcore <= 0.0 || rcore > rshell) inperr = 1;
  if (rindsh.re <= 0.0 || rindsh.im > 0.0) inperr = 1;
  if (rindco.re <= 0.0 || rindco.im > 0.0) inperr = 1;
  if (numang < 0 || numang > DM_MXANG) inperr = 1;
  if (nmx1 + 1 > DM_LL) inperr = 1;
  for (int j = 0; j < numang; ++j)
    if (mu[j] < -1.0e-6 || mu[j] > 1.0 + 1.0e-6) inperr = 1;
  if (inperr) return 1;

  cx k1 = cx_scale(wvno, rindco);
  cx k2 = cx_scale(wvno, rindsh);
  cx k3 = cx_make(wvno, 0.0);
  cx z[5];
  z[1] = cx_scale(xshell, rindsh);
  z[2] = cx_make(xshell, 0.0);
  z[3] = cx_scale(xcore, rindco);
  z[4] = cx_scale(xcore, rindsh);
  double x1 = z[1].re, y1 = z[1].im, x4 = z[4].re, y4 = z[4].im;
  double rx = 1.0 / xshell;

  /* down-recurrences for A and W (ComputePart.f:1439-1454) */
  cx *acap = (cx *)malloc(sizeof(cx) * (size_t)(nmx1 + 2));
  cx *w = (cx *)malloc(sizeof(cx) * 3 * (size_t)(nmx1 + 2)); /* w[(m-1)*(nmx1+2) + nn] */
  const size_t ws = (size_t)(nmx1 + 2);
  acap[nmx1 + 1] = cx_make(0.0, 0.0);
  for (int m = 0; m < 3; ++m) w[m * ws + nmx1 + 1] = cx_make(0.0, 0.0);
  cx rrfx = cx_rdiv(1.0, cx_scale(xshell, rindsh));
  for (int nn = nmx1; nn >= 1; --nn) {
    cx a = cx_scale((double)(nn + 1), rrfx);
    acap[nn] = cx_sub(a, cx_rdiv(1.0, cx_add(a, acap[nn + 1])));
    for (int m = 0; m < 3; ++m) {
      cx b = cx_rdiv((double)(nn + 1), z[m + 2]);
      w[m * ws + nn] = cx_sub(b, cx_rdiv(1.0, cx_add(b, w[m * ws + nn + 1])));
    }
  }
#define W1(n) w[0 * ws + (n)]
#define W2(n) w[1 * ws + (n)]
#define W3(n) w[2 * ws + (n)]

  double pi_[DM_MXANG][3], tau[DM_MXANG][3], si2tht[DM_MXANG];
  cx s1[DM_MXANG][2], s2[DM_MXANG][2];
  for (int j = 0; j < numang; ++j) {
    si2tht[j] = 1.0 - mu[j] * mu[j];
    pi_[j][0] = 0.0;
    pi_[j][1] = 1.0;
    tau[j][0] = 0.0;
    tau[j][1] = mu[j];
  }

  /* homogeneous sphere start (ComputePart.f:1469-1478) */
  double t[6], ta[5];
  t[1] = dm_cos(xshell);
  t[2] = dm_sin(xshell);
  cx wm1 = cx_make(t[1], -t[2]);
  cx wfn1 = cx_make(t[2], t[1]);
  ta[1] = t[2];
  ta[2] = t[1];
  cx wfn2 = cx_sub(cx_scale(rx, wfn1), wm1);
  ta[3] = wfn2.re;
  ta[4] = wfn2.im;

  /* stratified sphere start (ComputePart.f:1480-1530) */
  int n = 1;
  double sinx1 = dm_sin(x1), sinx4 = dm_sin(x4), cosx1 = dm_cos(x1), cosx4 = dm_cos(x4);
  double ey1 = dm_exp(y1);
  double e2y1 = ey1 * ey1;
  double ey4 = dm_exp(y4);
  double ey1my4 = dm_exp(y1 - y4);
  double ey1py4 = ey1 * ey4;
  double aa = sinx4 * (ey1py4 + ey1my4);
  double bb = cosx4 * (ey1py4 - ey1my4);
  double cc = sinx1 * (e2y1 + 1.0);
  double dd = cosx1 * (e2y1 - 1.0);
  double denom = 1.0 + e2y1 * ((4.0 * (sinx1 * sinx1) - 2.0) + e2y1);
  cx dummy = cx_make((aa * cc + bb * dd) / denom, (bb * cc - aa * dd) / denom);
  cx nz1 = cx_rdiv((double)n, z[1]);
  cx nz4 = cx_rdiv((double)n, z[4]);
  dummy = cx_div(cx_mul(dummy, cx_add(acap[n], nz1)), cx_add(W3(n), nz4));
  cx dumsq = cx_mul(dummy, dummy);
  cx p24h24 = cx_scale(ey4 * ey4, cx_make(sinx4 * sinx4 - 0.5, cosx4 * sinx4));
  p24h24 = cx_make(0.5 + p24h24.re, p24h24.im);
  cx p24h21 = cx_add(
      cx_scale(ey1py4, cx_scale(0.5, cx_make(sinx1 * sinx4 - cosx1 * cosx4,
                                             sinx1 * cosx4 + cosx1 * sinx4))),
      cx_scale(ey1my4, cx_scale(0.5, cx_make(sinx1 * sinx4 + cosx1 * cosx4,
                                             -(sinx1 * cosx4) + cosx1 * sinx4))));
  cx one = cx_make(1.0, 0.0);
  cx dh1 = cx_sub(cx_div(z[1], cx_add(one, cx_mul(CI, z[1]))), cx_rdiv(1.0, z[1]));
  cx dh2 = cx_sub(cx_div(z[2], cx_add(one, cx_mul(CI, z[2]))), cx_rdiv(1.0, z[2]));
  cx dh4 = cx_sub(cx_div(z[4], cx_add(one, cx_mul(CI, z[4]))), cx_rdiv(1.0, z[4]));
  p24h24 = cx_div(p24h24, cx_mul(cx_add(dh4, nz4), cx_add(W3(n), nz4)));
  p24h21 = cx_div(p24h21, cx_mul(cx_add(dh1, nz1), cx_add(W3(n), nz4)));

  cx u[9];
  u[1] = cx_sub(cx_mul(k3, acap[n]), cx_mul(k2, W1(n)));
  u[2] = cx_sub(cx_mul(k3, acap[n]), cx_mul(k2, dh2));
  u[3] = cx_sub(cx_mul(k2, acap[n]), cx_mul(k3, W1(n)));
  u[4] = cx_sub(cx_mul(k2, acap[n]), cx_mul(k3, dh2));
  u[5] = cx_sub(cx_mul(k1, W3(n)), cx_mul(k2, W2(n)));
  u[6] = cx_sub(cx_mul(k2, W3(n)), cx_mul(k1, W2(n)));
  u[7] = cx_neg(cx_mul(CI, cx_sub(cx_mul(dummy, p24h21), p24h24)));
  u[8] = cx_rdiv(ta[3], wfn2);

  cx acoe = cx_div(
      cx_mul(u[8], cx_sub(cx_add(cx_mul(cx_mul(u[1], u[5]), u[7]), cx_mul(k1, u[1])),
                          cx_mul(cx_mul(dumsq, k3), u[5]))),
      cx_sub(cx_add(cx_mul(cx_mul(u[2], u[5]), u[7]), cx_mul(k1, u[2])),
             cx_mul(cx_mul(dumsq, k3), u[5])));
  cx bcoe = cx_div(
      cx_mul(u[8], cx_sub(cx_add(cx_mul(cx_mul(u[3], u[6]), u[7]), cx_mul(k2, u[3])),
                          cx_mul(cx_mul(dumsq, k2), u[6]))),
      cx_sub(cx_add(cx_mul(cx_mul(u[4], u[6]), u[7]), cx_mul(k2, u[4])),
             cx_mul(cx_mul(dumsq, k2), u[6])));
  cx acoem1 = acoe, bcoem1 = bcoe;
  double are = acoe.re, aim = acoe.im, bre = bcoe.re, bim = bcoe.im;
  double dqext = 3.0 * (are + bre);
  double dqsca = 3.0 * (((are * are + aim * aim) + bre * bre) + bim * bim);
  double dgqsc = 0.0;
  cx sback = cx_scale(3.0, cx_sub(acoe, bcoe));
  double rmm = 1.0;
  cx ac = cx_scale(1.5, acoe);
  cx bc = cx_scale(1.5, bcoe);
  for (int j = 0; j < numang; ++j) {
    cx ap = cx_scale(pi_[j][1], ac), bt = cx_scale(tau[j][1], bc);
    cx bp = cx_scale(pi_[j][1], bc), at = cx_scale(tau[j][1], ac);
    s1[j][0] = cx_add(ap, bt);
    s1[j][1] = cx_sub(ap, bt);
    s2[j][0] = cx_add(bp, at);
    s2[j][1] = cx_sub(bp, at);
  }

  /* Mie summing loop (ComputePart.f:1545-1665) */
  int err = 0;
  n = 2;
  for (;;) {
    t[1] = (double)(2 * n - 1);
    t[2] = (double)(n - 1);
    for (int j = 0; j < numang; ++j) {
      pi_[j][2] = ((t[1] * pi_[j][1]) * mu[j] - (double)n * pi_[j][0]) / t[2];
      tau[j][2] = (mu[j] * (pi_[j][2] - pi_[j][0]) - (t[1] * si2tht[j]) * pi_[j][1]) + tau[j][0];
    }
    wm1 = wfn1;
    wfn1 = wfn2;
    wfn2 = cx_sub(cx_scale(t[1] * rx, wfn1), wm1);
    ta[1] = wfn1.re;
    ta[2] = wfn1.im;
    ta[3] = wfn2.re;
    ta[4] = wfn2.im;

    nz1 = cx_rdiv((double)n, z[1]);
    cx nz2 = cx_rdiv((double)n, z[2]);
    nz4 = cx_rdiv((double)n, z[4]);
    dh1 = cx_add(cx_neg(nz1), cx_rdiv(1.0, cx_sub(nz1, dh1)));
    dh2 = cx_add(cx_neg(nz2), cx_rdiv(1.0, cx_sub(nz2, dh2)));
    dh4 = cx_add(cx_neg(nz4), cx_rdiv(1.0, cx_sub(nz4, dh4)));
    p24h24 = cx_div(p24h24, cx_mul(cx_add(dh4, nz4), cx_add(W3(n), nz4)));
    p24h21 = cx_div(p24h21, cx_mul(cx_add(dh1, nz1), cx_add(W3(n), nz4)));
    dummy = cx_div(cx_mul(dummy, cx_add(acap[n], nz1)), cx_add(W3(n), nz4));
    dumsq = cx_mul(dummy, dummy);

    u[1] = cx_sub(cx_mul(k3, acap[n]), cx_mul(k2, W1(n)));
    u[2] = cx_sub(cx_mul(k3, acap[n]), cx_mul(k2, dh2));
    u[3] = cx_sub(cx_mul(k2, acap[n]), cx_mul(k3, W1(n)));
    u[4] = cx_sub(cx_mul(k2, acap[n]), cx_mul(k3, dh2));
    u[5] = cx_sub(cx_mul(k1, W3(n)), cx_mul(k2, W2(n)));
    u[6] = cx_sub(cx_mul(k2, W3(n)), cx_mul(k1, W2(n)));
    u[7] = cx_neg(cx_mul(CI, cx_sub(cx_mul(dummy, p24h21), p24h24)));
    u[8] = cx_rdiv(ta[3], wfn2);

    acoe = cx_div(
        cx_mul(u[8], cx_sub(cx_add(cx_mul(cx_mul(u[1], u[5]), u[7]), cx_mul(k1, u[1])),
                            cx_mul(cx_mul(dumsq, k3), u[5]))),
        cx_sub(cx_add(cx_mul(cx_mul(u[2], u[5]), u[7]), cx_mul(k1, u[2])),
               cx_mul(cx_mul(dumsq, k3), u[5])));
    bcoe = cx_div(
        cx_mul(u[8], cx_sub(cx_add(cx_mul(cx_mul(u[3], u[6]), u[7]), cx_mul(k2, u[3])),
                            cx_mul(cx_mul(dumsq, k2), u[6]))),
        cx_sub(cx_add(cx_mul(cx_mul(u[4], u[6]), u[7]), cx_mul(k2, u[4])),
               cx_mul(cx_mul(dumsq, k2), u[6])));
    are = acoe.re;
    aim = acoe.im;
    bre = bcoe.re;
    bim = bcoe.im;

    double am1re = acoem1.re, am1im = acoem1.im, bm1re = bcoem1.re, bm1im = bcoem1.im;
    double dn = (double)n;
    t[4] = ((double)(2 * n) - 1.0) / (dn * (dn - 1.0));
    t[2] = ((dn - 1.0) * (dn + 1.0)) / dn;
    dgqsc = (dgqsc + t[2] * (((am1re * are + am1im * aim) + bm1re * bre) + bm1im * bim)) +
            t[4] * (am1re * bm1re + am1im * bm1im);
    t[3] = (double)(2 * n + 1);
    dqext = dqext + t[3] * (are + bre);
    t[4] = ((are * are + aim * aim) + bre * bre) + bim * bim;
    dqsca = dqsca + t[3] * t[4];
    rmm = -rmm;
    sback = cx_add(sback, cx_scale(t[3] * rmm, cx_sub(acoe, bcoe)));
    t[2] = (double)(n * (n + 1));
    t[1] = t[3] / t[2];
    ac = cx_scale(t[1], acoe);
    bc = cx_scale(t[1], bcoe);
    for (int j = 0; j < numang; ++j) {
      cx ap = cx_scale(pi_[j][2], ac), bt = cx_scale(tau[j][2], bc);
      cx bp = cx_scale(pi_[j][2], bc), at = cx_scale(tau[j][2], ac);
      s1[j][0] = cx_add(cx_add(s1[j][0], ap), bt);
      s2[j][0] = cx_add(cx_add(s2[j][0], bp), at);
      if ((n & 1) == 0) {
        s1[j][1] = cx_add(cx_sub(s1[j][1], ap), bt);
        s2[j][1] = cx_add(cx_sub(s2[j][1], bp), at);
      } else {
        s1[j][1] = cx_sub(cx_add(s1[j][1], ap), bt);
        s2[j][1] = cx_sub(cx_add(s2[j][1], bp), at);
      }
    }
    if (t[4] >= 1.0e-14) {
      n = n + 1;
      if (n > nmx2) {
        err = 1;
        break;
      }
      for (int j = 0; j < numang; ++j) {
        pi_[j][0] = pi_[j][1];
        pi_[j][1] = pi_[j][2];
        tau[j][0] = tau[j][1];
        tau[j][1] = tau[j][2];
      }
      acoem1 = acoe;
      bcoem1 = bcoe;
      continue;
    }
    break;
  }
  free(acap);
  free(w);
#undef W1
#undef W2
#undef W3
  if (err) return 1;

  for (int j = 0; j < numang; ++j) {
    for (int k = 0; k < 2; ++k) {
      cx a = s1[j][k], b = s2[j][k];
      m1[k * numang + j] = a.re * a.re + a.im * a.im;
      m2[k * numang + j] = b.re * b.re + b.im * b.im;
      s21[k * numang + j] = a.re * b.re + a.im * b.im;
      d21[k * numang + j] = a.im * b.re - b.im * a.re;
    }
  }
  t[1] = 2.0 * (rx * rx);
  *qext = t[1] * dqext;
  *qsca = t[1] * dqsca;
  *gqsc = (2.0 * t[1]) * dgqsc;
  sback = cx_scale(0.5, sback);
  *qbs = (sback.re * sback.re + sback.im * sback.im) / (PI_D * (xshell * xshell));
  return 0;
}

/* ---------------------------------------------------------------- Mie */

int orc_meerhoff_mie(double rad, double lam, double e1, double e2, double *csca, double *cext,
                     double *f11, double *f12, double *f33, double *f34, int na) {
  /* MeerhoffMie sets thmin = 0.5, thmax = 179.5, step = 1 for na = 180 and a
   * single radius (idis = 0), so scatmat runs its symmetric branch. */
  if (na != ORC_NA) return 1;
  const int nangle = ORC_NA;
  const double pie = PI_D;
  const double radfac = pie / 180.0;
  const double rtox = 2.0 * pie / lam;
  const double fakt = lam * lam / (2.0 * pie);
  cx m = cx_make(e1, -e2);
  double x = rtox * rad;
  int nmax = (int)(x + 4.05 * dm_cbrt_pos(x) + 20.0);
  int nfi = nmax + 60;
  double zabs = x * cx_abs(m);
  int nD = (int)(zabs + 4.05 * dm_cbrt_pos(zabs) + 70.0);
  if (nD < nmax || nmax < 2) return 1;
  int nalloc = nD;
  if (nfi > nalloc) nalloc = nfi;
  double *psi = (double *)malloc(sizeof(double) * (size_t)(nalloc + 2));
  double *chi = (double *)malloc(sizeof(double) * (size_t)(nalloc + 2));
  cx *D = (cx *)malloc(sizeof(cx) * (size_t)(nalloc + 2));
  cx *an = (cx *)malloc(sizeof(cx) * (size_t)(nalloc + 2));
  cx *bn = (cx *)malloc(sizeof(cx) * (size_t)(nalloc + 2));
  double *pin = (double *)malloc(sizeof(double) * (size_t)(nalloc + 2));
  double *taun = (double *)malloc(sizeof(double) * (size_t)(nalloc + 2));
  double *facf = (double *)malloc(sizeof(double) * (size_t)(nalloc + 2));
  double *facb = (double *)malloc(sizeof(double) * (size_t)(nalloc + 2));

  /* fichid, ComputePart.f:2506-2560 */
  {
    cx zz = cx_scale(x, m);
    cx perz = cx_rdiv(1.0, zz);
    double perx = 1.0 / x;
    double sinx = dm_sin(x), cosx = dm_cos(x);
    psi[nfi] = 0.0;
    for (int k = nfi - 1; k >= 0; --k) psi[k] = 1.0 / ((double)(2 * k + 1) / x - psi[k + 1]);
    D[nD] = cx_make(0.0, 0.0);
    for (int k = nD - 1; k >= 1; --k) {
      cx zn1 = cx_scale((double)(k + 1), perz);
      D[k] = cx_sub(zn1, cx_rdiv(1.0, cx_add(D[k + 1], zn1)));
    }
    psi[0] = sinx;
    double psi1 = psi[0] * perx - cosx;
    if (fabs(psi1) > 1.0e-4) {
      psi[1] = psi1;
      for (int k = 2; k <= nmax; ++k) psi[k] = psi[k] * psi[k - 1];
    } else {
      for (int k = 1; k <= nmax; ++k) psi[k] = psi[k] * psi[k - 1];
    }
    chi[0] = cosx;
    chi[1] = chi[0] * perx + sinx;
    for (int k = 1; k <= nmax - 1; ++k)
      chi[k + 1] = ((double)(2 * k + 1) * chi[k]) * perx - chi[k - 1];
  }
  /* anbn, ComputePart.f:2211-2236 */
  {
    cx perm = cx_rdiv(1.0, m);
    double perx = 1.0 / x;
    for (int k = 1; k <= nmax; ++k) {
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
  for (int k = 1; k <= nmax; ++k) {
    facf[k] = (double)(2 * k + 1) / (double)(k * (k + 1));
    facb[k] = (k & 1) ? -facf[k] : facf[k];
  }
  /* cross sections and the truncation index (scatmat :2995-3010) */
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
  int nfou = nstop;
  /* scattering angles: u(nangle+1-iang) = cos(radfac*(0.5 + (iang-1))) */
  double uu[ORC_NA + 1];
  for (int iang = 1; iang <= nangle; ++iang) {
    double th = 0.5 + (double)(iang - 1) * 1.0;
    uu[nangle + 1 - iang] = dm_cos(radfac * th);
  }
  double F[4][ORC_NA + 1];
  memset(F, 0, sizeof F);
  const double sw = 1.0;
  int nhalf = nangle / 2;
  for (int j = 1; j <= nhalf; ++j) {
    /* pitau, ComputePart.f:2719-2740 */
    double uj = uu[j];
    pin[1] = 1.0;
    pin[2] = 3.0 * uj;
    double delta = (3.0 * uj) * uj - 1.0;
    taun[1] = uj;
    taun[2] = 2.0 * delta - 1.0;
    for (int k = 2; k <= nmax - 1; ++k) {
      pin[k + 1] = ((double)(k + 1) / (double)k) * delta + uj * pin[k];
      delta = uj * pin[k + 1] - pin[k];
      taun[k + 1] = (double)(k + 1) * delta - pin[k];
    }
    cx spf = cx_make(0, 0), smf = cx_make(0, 0), spb = cx_make(0, 0), smb = cx_make(0, 0);
    for (int k = 1; k <= nfou; ++k) {
      cx apb = cx_add(an[k], bn[k]);
      cx amb = cx_sub(an[k], bn[k]);
      double ppt = pin[k] + taun[k], pmt = pin[k] - taun[k];
      spf = cx_add(spf, cx_scale(ppt, cx_scale(facf[k], apb)));
      smf = cx_add(smf, cx_scale(pmt, cx_scale(facf[k], amb)));
      spb = cx_add(spb, cx_scale(pmt, cx_scale(facb[k], apb)));
      smb = cx_add(smb, cx_scale(ppt, cx_scale(facb[k], amb)));
    }
    cx cspf = cx_conj(spf), csmf = cx_conj(smf), cspb = cx_conj(spb), csmb = cx_conj(smb);
    int kk = nangle - j + 1;
    cx a, b;
    a = cx_mul(spf, cspf); b = cx_mul(smf, csmf);
    F[0][j] = F[0][j] + sw * (a.re + b.re);
    F[2][j] = F[2][j] + sw * (a.re - b.re);
    a = cx_mul(smf, cspf); b = cx_mul(spf, csmf);
    F[1][j] = F[1][j] - sw * (a.re + b.re);
    F[3][j] = F[3][j] + (0.0 * (a.re - b.re) - sw * (a.im - b.im));
    a = cx_mul(spb, cspb); b = cx_mul(smb, csmb);
    F[0][kk] = F[0][kk] + sw * (a.re + b.re);
    F[2][kk] = F[2][kk] + sw * (a.re - b.re);
    a = cx_mul(smb, cspb); b = cx_mul(spb, csmb);
    F[1][kk] = F[1][kk] - sw * (a.re + b.re);
    F[3][kk] = F[3][kk] + (0.0 * (a.re - b.re) - sw * (a.im - b.im));
  }
  double Csca = sw * cscasum;
  double Cext = sw * cextsum;
  for (int j = 1; j <= nangle; ++j)
    for (int k = 0; k < 4; ++k) F[k][j] = F[k][j] / (2.0 * Csca);
  Csca = Csca * fakt;
  Cext = Cext * fakt;
  *csca = Csca;
  *cext = Cext;
  for (int i = 1; i <= nangle; ++i) {
    f11[i - 1] = F[0][nangle - i + 1];
    f12[i - 1] = F[1][nangle - i + 1];
    f33[i - 1] = F[2][nangle - i + 1];
    f34[i - 1] = F[3][nangle - i + 1];
  }
  free(psi); free(chi); free(D); free(an); free(bn);
  free(pin); free(taun); free(facf); free(facb);
  return 0;
}

/* ---------------------------------------------------------------- Blender */

void orc_blender(const double *e1, const double *e2, const double *abun, int nm, double *e1out,
                 double *e2out) {
  cx mm = cx_make(1.0, 0.0), me = mm;
  for (int iter = 0; iter < 100; ++iter) {
    cx sum = cx_make(0.0, 0.0);
    cx mm2 = cx_mul(mm, mm);
    for (int j = 0; j < nm; ++j) {
      cx mj = cx_make(e1[j], e2[j]);
      cx mj2 = cx_mul(mj, mj);
      cx q = cx_div(cx_sub(mj2, mm2), cx_add(mj2, cx_scale(2.0, mm2)));
      sum = cx_add(sum, cx_scale(abun[j], q));
    }
    cx num = cx_make(2.0 * sum.re + 1.0, 2.0 * sum.im);
    cx den = cx_make(1.0 - sum.re, -sum.im);
    me = cx_div(num, den);
    me = cx_mul(mm, cx_sqrt(me));
    mm = me;
  }
  *e1out = me.re;
  *e2out = me.im;
}

/* ---------------------------------------------------------------- gauleg2 */

void orc_gauleg2(double x1, double x2, double *x, double *w, int n) {
  int m = (n + 1) / 2;
  double xm = 0.5 * (x2 + x1);
  double xl = 0.5 * (x2 - x1);
  for (int i = 1; i <= m; ++i) {
    double z = cos(3.141592654 * ((double)i - 0.25) / ((double)n + 0.5));
    double z1, pp;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= n; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (!(fabs(z - z1) > 3.0e-14)) break;
    }
    x[i - 1] = xm - xl * z;
    x[n - i] = xm + xl * z;
    w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

/* ---------------------------------------------------------------- ComputePart */

int orc_compute_part(int nlam, const double *lam, int nm, const double *e1in, const double *e2in,
                     const double *frac_in, const double *rho_in, double amin, double amax,
                     double apow, double fmax, int blend, double porosity, int ns, int nf,
                     double normalize_abun, double *kabs, double *ksca, double *kext, double *Fout,
                     double *rho_av_out, double *mscale_out, double *rscale_out,
                     int64_t *counters) {
  if (nlam < 1 || nm < 1 || ns < 1 || nf < 1 || amin <= 0.0 || amax <= 0.0) return -1;
  const int na = ORC_NA;
  int nmat = nm + (blend ? 1 : 0);
  double *e1 = (double *)malloc(sizeof(double) * (size_t)nmat * (size_t)nlam);
  double *e2 = (double *)malloc(sizeof(double) * (size_t)nmat * (size_t)nlam);
  double *frac = (double *)malloc(sizeof(double) * (size_t)nmat);
  double *rho = (double *)malloc(sizeof(double) * (size_t)nmat);
  memcpy(e1, e1in, sizeof(double) * (size_t)nm * (size_t)nlam);
  memcpy(e2, e2in, sizeof(double) * (size_t)nm * (size_t)nlam);
  for (int l = 0; l < nm; ++l) {
    rho[l] = rho_in[l];
    frac[l] = frac_in[l] / rho_in[l]; /* mass fractions -> volume, ComputePart.f:85 */
  }
  double minlog = log10(amin), maxlog = log10(amax);
  double pw = -apow;
  double maxf = fmax;
  if (maxf == 0.0) nf = 1; /* ComputePart.f:70 */

  /* abundance normalisation and radius/mass scaling, ComputePart.f:139-156 */
  double tot = 0.0;
  for (int i = 0; i < nm; ++i) tot += frac[i];
  double mscale, rscale;
  if (normalize_abun <= 0.0) {
    for (int i = 0; i < nm; ++i) frac[i] /= tot;
    mscale = 1.0;
    rscale = 1.0;
  } else {
    mscale = 0.0;
    for (int i = 0; i < nm; ++i) mscale += frac[i] * rho[i] / normalize_abun;
    rscale = pow(mscale, 1.0 / 3.0);
    for (int i = 0; i < nm; ++i) frac[i] /= tot;
  }

  /* porous blend with vacuum, ComputePart.f:227-252 */
  int nmc = nm;
  if (blend) {
    nmc = nm + 1;
    for (int i = 0; i < nlam; ++i) {
      e1[(size_t)nm * nlam + i] = 1.0;
      e2[(size_t)nm * nlam + i] = 0.0;
    }
    rho[nm] = 0.0;
    frac[nm] = porosity;
    for (int l = 0; l < nm; ++l) frac[l] *= (1.0 - porosity);
    double ee1[64], ee2[64];
    if (nmc > 64) { free(e1); free(e2); free(frac); free(rho); return -1; }
    for (int i = 0; i < nlam; ++i) {
      for (int l = 0; l < nmc; ++l) {
        ee1[l] = e1[(size_t)l * nlam + i];
        ee2[l] = e2[(size_t)l * nlam + i];
      }
      double b1, b2;
      orc_blender(ee1, ee2, frac, nmc, &b1, &b2);
      e1[i] = b1;
      e2[i] = b2;
    }
    double rav = 0.0;
    for (int l = 0; l < nmc; ++l) rav += frac[l] * rho[l];
    rho[0] = rav;
    frac[0] = 1.0;
    nmc = 1;
  }

  /* filling-fraction nodes, ComputePart.f:266-274 */
  double *f = (double *)malloc(sizeof(double) * (size_t)nf);
  double *wf = (double *)malloc(sizeof(double) * (size_t)nf);
  if (nf > 1 && maxf > 0.01) {
    orc_gauleg2(0.01, maxf, f, wf, nf);
  } else if (maxf == 0.0) {
    for (int i = 0; i < nf; ++i) {
      f[i] = 0.0;
      wf[i] = 1.0 / (double)nf;
    }
  } else {
    nf = 1; /* the reference leaves f(2:nf) undefined here; use one node */
    f[0] = maxf;
    wf[0] = 1.0;
  }

  /* size grid and number weights, ComputePart.f:276-292 */
  double *r = (double *)malloc(sizeof(double) * (size_t)ns);
  double *nr = (double *)malloc(sizeof(double) * (size_t)nmc * (size_t)ns);
  for (int l = 0; l < nmc; ++l) {
    if (ns == 1) {
      r[0] = pow(10.0, (minlog + maxlog) / 2.0);
      nr[l * ns] = frac[l];
    } else {
      double t2 = 0.0;
      for (int k = 0; k < ns; ++k) {
        r[k] = pow(10.0, minlog + (maxlog - minlog) * (double)k / (double)(ns - 1));
        nr[l * ns + k] = pow(r[k], pw + 1.0);
        t2 += nr[l * ns + k] * (r[k] * r[k] * r[k]);
      }
      for (int k = 0; k < ns; ++k) nr[l * ns + k] = frac[l] * nr[l * ns + k] / t2;
    }
  }

  /* DHS angles mu(i) = cos((i-1/2)/90 * pi/2), ComputePart.f:294-297 */
  double mu[ORC_NA / 2];
  for (int i = 1; i <= na / 2; ++i) mu[i - 1] = cos(((double)i - 0.5) / (double)(na / 2) * PI_D / 2.0);
  /* forward-peak renormalisation weights sin(pi (j-1/2)/na), :407-415 */
  double sinw[ORC_NA];
  for (int j = 1; j <= na; ++j) sinw[j - 1] = sin(PI_D * ((double)j - 0.5) / (double)na);

  double m1[ORC_NA], m2[ORC_NA], s21[ORC_NA], d21[ORC_NA];
  double mf11[ORC_NA], mf12[ORC_NA], mf22[ORC_NA], mf33[ORC_NA], mf34[ORC_NA], mf44[ORC_NA];
  double *acc = (double *)malloc(sizeof(double) * 6 * ORC_NA);
  int64_t n_dhs = 0, n_mie = 0, n_fail = 0;
  double rho_av = 0.0;

  for (int ilam = 0; ilam < nlam; ++ilam) {
    double csca = 0.0, cabs = 0.0, cext = 0.0, mass = 0.0, vol = 0.0;
    memset(acc, 0, sizeof(double) * 6 * ORC_NA);
    double csmie = 0.0, cemie = 0.0;
    for (int l = 0; l < nmc; ++l) {
      if (frac[l] == 0.0) continue;
      for (int k = 0; k < ns; ++k) {
        double r1 = r[k] * rscale;
        int err = 0;
        for (int i = 0; i < nf; ++i) {
          double rad = r1 / pow(1.0 - f[i], 1.0 / 3.0);
          double me1 = e1[(size_t)l * nlam + ilam], me2 = e2[(size_t)l * nlam + ilam];
          double wvno = 2.0 * PI_D / lam[ilam];
          int spheres = 0, toolarge = 0;
          double qext = 0, qsca = 0, qbs, gqsc;
          if (f[i] == 0.0) {
            spheres = 1;
          } else if (r1 * wvno > 10000.0) {
            toolarge = 1;
          } else {
            double rcore = rad * pow(f[i], 1.0 / 3.0);
            int e = orc_dmilay(rcore, rad, wvno, me1, -me2, 1.0, 0.0, mu, na / 2, &qext, &qsca,
                               &qbs, &gqsc, m1, m2, s21, d21);
            n_dhs++;
            if (e) {
              err = 1;
              n_fail++;
            }
          }
          if (err || spheres || toolarge) {
            rad = r1;
            if (err || i == 0) {
              double rmie = rad, lmie = lam[ilam];
              if (rmie / lmie >= 5000.0) lmie = rmie / 5000.0;
              orc_meerhoff_mie(rmie, lmie, me1, me2, &csmie, &cemie, mf11, mf12, mf33, mf34, na);
              n_mie++;
            }
            for (int j = 0; j < na; ++j) {
              mf22[j] = mf11[j];
              mf44[j] = mf33[j];
            }
          } else {
            cemie = qext * PI_D * (rad * rad);
            csmie = qsca * PI_D * (rad * rad);
            double w2 = wvno * wvno;
            for (int j = 0; j < na / 2; ++j) {
              int jb = na - 1 - j;
              mf11[j] = (((m2[j] + m1[j]) / csmie) / w2) * 2.0 * PI_D;
              mf12[j] = (((m2[j] - m1[j]) / csmie) / w2) * 2.0 * PI_D;
              mf22[j] = mf11[j];
              mf33[j] = ((s21[j] / csmie) / w2) * 2.0 * PI_D;
              mf34[j] = ((-d21[j] / csmie) / w2) * 2.0 * PI_D;
              mf44[j] = mf33[j];
              int q = na / 2 + j;
              mf11[jb] = (((m2[q] + m1[q]) / csmie) / w2) * 2.0 * PI_D;
              mf12[jb] = (((m2[q] - m1[q]) / csmie) / w2) * 2.0 * PI_D;
              mf22[jb] = mf11[jb];
              mf33[jb] = ((s21[q] / csmie) / w2) * 2.0 * PI_D;
              mf34[jb] = ((-d21[q] / csmie) / w2) * 2.0 * PI_D;
              mf44[jb] = mf33[jb];
            }
          }
          /* forward-peak renormalisation, ComputePart.f:407-415 */
          double t1 = 0.0, t2 = 0.0;
          for (int j = 0; j < na; ++j) {
            t1 = t1 + mf11[j] * sinw[j];
            t2 = t2 + sinw[j];
          }
          mf11[0] = mf11[0] + (t2 - t1) / sinw[0];
          if (mf11[0] < 0.0) mf11[0] = 0.0;
          double wn = wf[i] * nr[l * ns + k];
          for (int j = 0; j < na; ++j) {
            acc[0 * na + j] += (wn * mf11[j]) * csmie;
            acc[1 * na + j] += (wn * mf12[j]) * csmie;
            acc[2 * na + j] += (wn * mf22[j]) * csmie;
            acc[3 * na + j] += (wn * mf33[j]) * csmie;
            acc[4 * na + j] += (wn * mf34[j]) * csmie;
            acc[5 * na + j] += (wn * mf44[j]) * csmie;
          }
          cext = cext + wn * cemie;
          csca = csca + wn * csmie;
          cabs = cabs + wn * (cemie - csmie);
          double r13 = (r1 * r1) * r1;
          mass = mass + (((wn * rho[l]) * 4.0) * PI_D) * r13 / 3.0;
          vol = vol + ((wn * 4.0) * PI_D) * r13 / 3.0;
        }
      }
    }
    rho_av = mass / vol;
    kabs[ilam] = 1.0e4 * cabs / (mass / mscale);
    ksca[ilam] = 1.0e4 * csca / (mass / mscale);
    kext[ilam] = 1.0e4 * cext / (mass / mscale);
    for (int b = 0; b < 6; ++b)
      for (int j = 0; j < na; ++j) Fout[((size_t)ilam * 6 + b) * na + j] = acc[b * na + j] / csca;
  }
  *rho_av_out = rho_av;
  *mscale_out = mscale;
  *rscale_out = rscale;
  if (counters) {
    counters[0] = n_dhs;
    counters[1] = n_mie;
    counters[2] = n_fail;
  }
  free(acc); free(e1); free(e2); free(frac); free(rho); free(f); free(wf); free(r); free(nr);
  return 0;
}
