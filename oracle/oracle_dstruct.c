/*
 * oracle_dstruct.c -- CPU restatement of the vertical structure step
 * (DiskStructure, DiskStructure.f:85-468, with CheckMinimumDensity
 * DiskStructure.f:2966 and CheckCells DiskStructure.f:2659), test
 * infrastructure only: the checker of mcg_disk_structure, never linked by
 * the product.
 *
 * Loop order and arithmetic as the reference: ring by ring, gas (ii = 0)
 * then each grain, the column integrated from the midplane to the pole with
 * odeint/rkqs/rkck (Subroutines.f:1933-2090, every stage formed as there;
 * derivs ignores y) and the constants at their widened single-precision
 * values; then the cells of the ring.  exp and log, and the powers of the
 * step-size control and the fixed-zone profile, are the deterministic
 * functions of detmath.h (the reference calls libm; they differ in the last
 * bits).  Grains of the other scale-height types take the closed-form
 * profiles of DiskStructure.f:248-344 (ZODI, HALO, LOBE, JET, SHELL, CYLI,
 * CAVITY, WEDGE, an unknown type keeping log(dens w)), formed with the C
 * library's functions; D%thet(j) is taken as acos(Theta(j)).  No radiation
 * pressure, gaps, halo or radial iterations.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "oracle.h"
#include "../mcmax_b200/csrc/detmath.h"

#define AU_D ((double)1.49598e13f)
#define PI_D 3.14159265358979323846

typedef struct {
  double z1, z2, T1, T2, Mstar, scale, Rav;
} seg_t;

/* derivs, DiskStructure.f:469-491 (beta = 0) */
static void derivs(const seg_t *s, double x, const double *y, double *dydx) {
  const double mu = (double)2.3f * 1.67262158e-24, G = 6.67300e-8, kb = 1.3806503e-16;
  (void)y;
  const double T = s->T1 + ((s->T2 - s->T1) * (x - s->z1)) / (s->z2 - s->z1);
  const double dlnT = (dm_log(s->T1) - dm_log(s->T2)) / (s->z1 - s->z2);
  const double beta = 0.0;
  dydx[0] = -((((mu * G) * s->Mstar) * (1.0 + beta)) * x) / ((((s->scale * s->scale) * kb) * T) * ((s->Rav * s->Rav) * s->Rav)) - dlnT;
}

static double pw(double x, double y) { return dm_exp(y * dm_log(x)); }

static void rkck(const seg_t *s, double y, double dydx, double x, double h, double *yout, double *yerr) {
  const double A2 = (double).2f, A3 = (double).3f, A4 = (double).6f, A5 = (double)1.f, A6 = (double).875f;
  const double B21 = (double).2f, B31 = (double)(3.f / 40.f), B32 = (double)(9.f / 40.f), B41 = (double).3f,
               B42 = (double)-.9f, B43 = (double)1.2f, B51 = (double)(-11.f / 54.f), B52 = (double)2.5f,
               B53 = (double)(-70.f / 27.f), B54 = (double)(35.f / 27.f), B61 = (double)(1631.f / 55296.f),
               B62 = (double)(175.f / 512.f), B63 = (double)(575.f / 13824.f), B64 = (double)(44275.f / 110592.f),
               B65 = (double)(253.f / 4096.f);
  const double C1 = (double)(37.f / 378.f), C3 = (double)(250.f / 621.f), C4 = (double)(125.f / 594.f),
               C6 = (double)(512.f / 1771.f);
  const double DC1 = C1 - (double)(2825.f / 27648.f), DC3 = C3 - (double)(18575.f / 48384.f),
               DC4 = C4 - (double)(13525.f / 55296.f), DC5 = (double)(-277.f / 14336.f), DC6 = C6 - (double).25f;
  double yt, ak2, ak3, ak4, ak5, ak6;
  yt = y + (B21 * h) * dydx;
  derivs(s, x + A2 * h, &yt, &ak2);
  yt = y + h * (B31 * dydx + B32 * ak2);
  derivs(s, x + A3 * h, &yt, &ak3);
  yt = y + h * ((B41 * dydx + B42 * ak2) + B43 * ak3);
  derivs(s, x + A4 * h, &yt, &ak4);
  yt = y + h * (((B51 * dydx + B52 * ak2) + B53 * ak3) + B54 * ak4);
  derivs(s, x + A5 * h, &yt, &ak5);
  yt = y + h * ((((B61 * dydx + B62 * ak2) + B63 * ak3) + B64 * ak4) + B65 * ak5);
  derivs(s, x + A6 * h, &yt, &ak6);
  *yout = y + h * (((C1 * dydx + C3 * ak3) + C4 * ak4) + C6 * ak6);
  *yerr = h * ((((DC1 * dydx + DC3 * ak3) + DC4 * ak4) + DC5 * ak5) + DC6 * ak6);
}

static void rkqs(const seg_t *s, double *y, double dydx, double *x, double htry, double eps, double yscal,
                 double *hdid, double *hnext) {
  const double SAFETY = (double)0.9f, PGROW = (double)-.2f, PSHRNK = (double)-.25f, ERRCON = (double)1.89e-4f;
  double h = htry, ytemp, yerr;
  for (int guard = 0; guard < 200; ++guard) {
    rkck(s, *y, dydx, *x, h, &ytemp, &yerr);
    double errmax = 0.0;
    if (fabs(yerr / yscal) > errmax) errmax = fabs(yerr / yscal);
    errmax = errmax / eps;
    if (errmax > 1.0) {
      double htemp = (SAFETY * h) * pw(errmax, PSHRNK);
      double a = fabs(htemp) > (double)0.1f * fabs(h) ? fabs(htemp) : (double)0.1f * fabs(h);
      h = copysign(a, h);
      continue;
    }
    *hnext = errmax > ERRCON ? (SAFETY * h) * pw(errmax, PGROW) : 5.0 * h;
    *hdid = h;
    *x = *x + h;
    *y = ytemp;
    return;
  }
  *hdid = h;
  *hnext = h;
  *x = *x + h;
}

static double odeint(const seg_t *s, double ystart, double eps, double h1) {
  const double x1 = s->z1, x2 = s->z2, TINY = 1.e-150;
  double x = x1, y = ystart, h = copysign(fabs(h1), x2 - x1), dydx, hdid, hnext;
  for (int nstp = 1; nstp <= 10000; ++nstp) {
    derivs(s, x, &y, &dydx);
    const double yscal = (fabs(y) + fabs(h * dydx)) + TINY;
    if (((x + h) - x2) * ((x + h) - x1) > 0.0) h = x2 - x;
    rkqs(s, &y, dydx, &x, h, eps, yscal, &hdid, &hnext);
    if ((x - x2) * (x2 - x1) >= 0.0) return y;
    h = hnext;
  }
  return y;
}

/* the closed-form profiles of DiskStructure.f:248-344 (types as
 * MCG_SH_*: 1 ZODI, 2 HALO, 3 LOBE, 4 JET, 5 SHELL, 6 CYLI, 7 CAVITY,
 * 8 WEDGE, 9 unknown), rho[1..nc] for grain ii of the ring; th, z 1-based
 * (theta_av, R_av cos theta_av), Theta the cos-theta edges, dw/wr the
 * ring's dens and abundance rows */
static void shape_profile(int type, int nc, double scale, double gsh, double Rav, double Rout, const double *th,
                          const double *Theta, const double *z, const double *dw, const double *wr, int ng, int ii,
                          double *rho) {
  const double pi = PI_D;
  switch (type) {
    case 1:
      for (int j = 1; j <= nc; ++j) rho[j] = log(0.15 + (double)0.85f * pow(cos(pi / 2.0 - th[j]), 28.0));
      break;
    case 2:
      for (int j = 1; j <= nc; ++j) {
        rho[j] = 0.0;
        if (gsh < 0.0 && pi / 2.0 - th[j] > -gsh) rho[j] = -60.0;
      }
      break;
    case 3:
      for (int j = 1; j <= nc; ++j) {
        const double a = ((th[j] * 180.0) / pi) / scale;
        rho[j] = log10(exp(-(a * a)));
      }
      break;
    case 4:
      for (int j = 1; j <= nc; ++j) {
        const double a = ((acos(Theta[j - 1]) * 180.0) / pi) / (scale * (Rav / Rout));
        rho[j] = -(a * a);
      }
      break;
    case 5:
      for (int j = 1; j <= nc; ++j) rho[j] = log(1.0 + gsh * pow(sin(th[j]), 3.0));
      break;
    case 6:
      rho[nc] = 0.0;
      for (int j = nc - 1; j >= 1; --j) rho[j] = (z[j] / AU_D < scale) ? 0.0 : -60.0;
      break;
    case 7:
      rho[nc] = 0.0;
      rho[1] = -60.0;
      for (int j = nc - 1; j >= 2; --j) {
        const double Rcyl = Rav * sin(th[j]);
        rho[j] = (z[j] / AU_D < ((Rcyl / AU_D) * (Rcyl / AU_D)) * scale) ? 0.0 : -60.0;
      }
      break;
    case 8:
      for (int j = 1; j <= nc; ++j) {
        if (scale > 0.0)
          rho[j] = ((180.0 * th[j]) / pi > scale) ? 0.0 : -60.0;
        else
          rho[j] = ((180.0 * th[j]) / pi < -scale) ? 0.0 : -60.0;
      }
      break;
    default:
      for (int j = 1; j <= nc; ++j) {
        const double v = dw[j - 1] * wr[(size_t)(j - 1) * ng + (ii - 1)];
        rho[j] = v > 1e-60 ? log(v) : -60.0;
      }
  }
}

int orc_disk_structure(int nR, int nTheta, int ng, const double *R, const double *Theta, const double *V,
                       double Mstar, int nzones, const double *zones, const double *shscale,
                       const double *grain_scale, const int *shtype, const double *Temp, double *dens,
                       double *dens0, double *gasdens, double *w, double *w0) {
  const int nc = nTheta - 1;
#define CI(i, j) ((size_t)(i) * nc + ((j) - 1))
  double *Rav = (double *)malloc(sizeof(double) * nR), *th = (double *)malloc(sizeof(double) * (nc + 1));
  double *z = (double *)malloc(sizeof(double) * (nc + 1));
  double *rho = (double *)malloc(sizeof(double) * (size_t)(nc + 1) * (ng + 1));
  double *M0 = (double *)malloc(sizeof(double) * (ng + 1)), *gasf = (double *)malloc(sizeof(double) * ng);
  double *tot = (double *)malloc(sizeof(double) * ng);
  for (int i = 0; i < nR; ++i) Rav[i] = AU_D * pow(10.0, (log10(R[i]) + log10(R[i + 1])) / 2.0);
  for (int j = 1; j <= nc; ++j) th[j] = acos((Theta[j - 1] + Theta[j]) / 2.0);
#define RHO(j, ii) rho[(size_t)(ii) * (nc + 1) + (j)]
  for (int i = 1; i <= nR - 1; ++i) {
    for (int ii = 0; ii <= ng; ++ii) {
      double scale;
      if (ii != 0) {
        scale = shscale ? shscale[i] : 1.0;
        if (grain_scale) scale = scale * grain_scale[(size_t)(ii - 1) * nR + i];
      } else {
        scale = 1.0 * (shscale ? shscale[i] : 1.0);
      }
      M0[ii] = 0.0;
      for (int j = 1; j <= nc; ++j) {
        if (ii != 0)
          M0[ii] = M0[ii] + (dens0[CI(i, j)] * V[CI(i, j)]) * w0[CI(i, j) * ng + (ii - 1)];
        else
          M0[ii] = M0[ii] + gasdens[CI(i, j)] * V[CI(i, j)];
        z[j] = Rav[i] * cos(th[j]);
      }
      int fix = -1;
      for (int iz = 0; iz < nzones; ++iz) {
        const double *zn = zones + 7 * iz; /* rin rout sh rsh shpow denspow fix_struct */
        if (Rav[i] > zn[0] * AU_D && Rav[i] < zn[1] * AU_D && zn[6] != 0.0) fix = iz;
      }
      if (ii == 0)
        for (int iz = 0; iz < nzones; ++iz) {
          const double *zn = zones + 7 * iz;
          if (Rav[i] > zn[0] * AU_D && Rav[i] < zn[1] * AU_D && zn[6] == 0.0) fix = -1;
        }
      const int type = (ii != 0 && shtype) ? shtype[ii - 1] : 0;
      if (fix < 0 && type != 0) {
        const double gsh = grain_scale ? grain_scale[(size_t)(ii - 1) * nR + i] : 1.0;
        shape_profile(type, nc, scale, gsh, Rav[i], Rav[nR - 1], th, Theta, z, dens + CI(i, 1), w + CI(i, 1) * ng,
                      ng, ii, &RHO(0, ii));
      } else if (fix < 0) {
        RHO(nc, ii) = 0.0;
        if (scale > 0.0) {
          for (int j = nc - 1; j >= 1; --j) {
            seg_t s = {z[j + 1], z[j], Temp[CI(i, j + 1)], Temp[CI(i, j)], Mstar, scale, Rav[i]};
            const double h1 = fabs(z[j] - z[j + 1]) * 1e-6;
            RHO(j, ii) = odeint(&s, RHO(j + 1, ii), 1e-6, h1);
          }
        } else {
          for (int j = nc - 1; j >= 1; --j) RHO(j, ii) = ((1.0 / tan(th[j])) < (-scale)) ? 0.0 : -60.0;
        }
      } else {
        const double *zn = zones + 7 * fix;
        if (zn[2] < 0.0) {
          RHO(nc, ii) = 0.0;
          for (int j = 1; j <= nc - 1; ++j) RHO(j, ii) = ((180.0 * th[j]) / PI_D > (-zn[2])) ? 0.0 : -60.0;
        } else {
          for (int j = 1; j <= nc; ++j) {
            const double rr = (Rav[i] * sin(th[j])) / AU_D, zz = (Rav[i] * cos(th[j])) / AU_D;
            const double hr = (scale * zn[2]) * pw(rr / zn[3], zn[4]);
            const double f1 = pw(rr, -zn[5]);
            double f2 = -((zz / hr) * (zz / hr));
            if (j == nc) f2 = 0.0;
            RHO(j, ii) = dm_log(f1 / hr) + f2;
          }
        }
      }
      double M1 = 0.0;
      for (int j = 1; j <= nc; ++j) M1 = M1 + dm_exp(RHO(j, ii)) * V[CI(i, j)];
      for (int j = 1; j <= nc; ++j) {
        RHO(j, ii) = (dm_exp(RHO(j, ii)) * M0[ii]) / M1;
        if (RHO(j, ii) < 1e-50) RHO(j, ii) = 1e-50;
      }
    }
    for (int j = 1; j <= nc; ++j) {
      const size_t c = CI(i, j);
      double *wc = w + c * ng, *w0c = w0 + c * ng;
      for (int ii = 0; ii < ng; ++ii) {
        if (w0c[ii] >= 1e-100)
          gasf[ii] = 1.0 - (dens[c] * wc[ii]) / (dens0[c] * w0c[ii]);
        else
          gasf[ii] = 0.0;
        if (gasf[ii] < 0.0) gasf[ii] = 0.0;
        if (gasf[ii] > 1.0) gasf[ii] = 1.0;
        if (isnan(gasf[ii])) gasf[ii] = 0.0;
      }
      gasdens[c] = RHO(j, 0);
      dens0[c] = 0.0;
      for (int ii = 1; ii <= ng; ++ii) dens0[c] = dens0[c] + RHO(j, ii);
      if (dens0[c] > 1e-50)
        for (int ii = 1; ii <= ng; ++ii) w0c[ii - 1] = RHO(j, ii) / dens0[c];
      double t = 0.0;
      for (int ii = 0; ii < ng; ++ii) t = t + w0c[ii];
      for (int ii = 0; ii < ng; ++ii) {
        w0c[ii] = w0c[ii] / t;
        wc[ii] = w0c[ii] * (1.0 - gasf[ii]);
      }
      t = 0.0;
      for (int ii = 0; ii < ng; ++ii) t = t + wc[ii];
      if (t > 1e-50)
        for (int ii = 0; ii < ng; ++ii) wc[ii] = wc[ii] / t;
      else
        for (int ii = 0; ii < ng; ++ii) wc[ii] = w0c[ii];
      dens[c] = dens0[c] * t;
      /* CheckMinimumDensity */
      if (dens0[c] <= 1e-50) dens0[c] = 1e-50;
      if (dens[c] <= 1e-50) dens[c] = 1e-50;
      if (gasdens[c] <= 1e-50) gasdens[c] = 1e-50;
      for (int ii = 0; ii < ng; ++ii) {
        tot[ii] = dens[c] * wc[ii];
        if (tot[ii] < 1e-50) tot[ii] = 1e-50;
        if (tot[ii] > dens0[c] * w0c[ii]) tot[ii] = dens0[c] * w0c[ii];
      }
      dens[c] = 0.0;
      for (int ii = 0; ii < ng; ++ii) dens[c] = dens[c] + tot[ii];
      if (dens[c] <= 1e-50) {
        dens[c] = 1e-50;
        for (int ii = 0; ii < ng; ++ii) wc[ii] = w0c[ii];
      } else {
        for (int ii = 0; ii < ng; ++ii) wc[ii] = tot[ii] / dens[c];
      }
    }
  }
  /* CheckCells over rings 0..nR-1 */
  for (int i = 0; i <= nR - 1; ++i)
    for (int j = 1; j <= nc; ++j) {
      const size_t c = CI(i, j);
      double *wc = w + c * ng, *w0c = w0 + c * ng;
      int rescale = 0;
      for (int ii = 0; ii < ng; ++ii) {
        tot[ii] = dens[c] * wc[ii];
        const double mx = dens0[c] * w0c[ii];
        if (tot[ii] > mx) {
          tot[ii] = mx;
          rescale = 1;
        }
      }
      if (rescale) {
        dens[c] = 0.0;
        for (int ii = 0; ii < ng; ++ii) dens[c] = dens[c] + tot[ii];
        if (dens[c] > 1e-50) {
          for (int ii = 0; ii < ng; ++ii) wc[ii] = tot[ii] / dens[c];
        } else {
          dens[c] = 1e-50;
          for (int ii = 0; ii < ng; ++ii) wc[ii] = w0c[ii];
        }
      }
    }
#undef RHO
#undef CI
  free(Rav); free(th); free(z); free(rho); free(M0); free(gasf); free(tot);
  return 0;
}
