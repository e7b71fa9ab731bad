/*
 * oracle_tables.c -- CPU restatement of the tables the MCMax packet loop
 * reads, plus the temperature inversions.  Test infrastructure only.
 *
 *   Planck        Subroutines.f:4-21  (quad-precision exponential)
 *   BB table      Init.f:2616-2622
 *   integrate     Radiation.f:1-18
 *   increaseT     Radiation.f:537-562
 *   determineT    Radiation.f:629-702
 *   ran1          Subroutines.f:1481-1509
 */
#include <math.h>
#include <quadmath.h>
#include <stdlib.h>
#include <stdint.h>

#include "oracle.h"

double orc_planck(double T, double lam) {
  const double k = 1.3807e-16, c = 2.9979e10, h = 6.6261e-27;
  double nu = c / (lam * 1e-4);
  double xd = (h * nu) / (k * T);
  __float128 x = (__float128)xd;
  if (x > (__float128)1e3) return 0.0;
  double num = ((2.0 * h) * ((nu * nu) * nu)) / (c * c);
  __float128 den = expq(x) - (__float128)1.0;
  return (double)((__float128)num / den);
}

void orc_bb_table(int nlam, const double *lam, double *BB) {
  for (int i = 0; i < nlam; ++i) {
    BB[(size_t)i * (ORC_TMAX + 1)] = 0.0;
    for (int j = 1; j <= ORC_TMAX; ++j) BB[(size_t)i * (ORC_TMAX + 1) + j] = orc_planck((double)j, lam[i]);
  }
}

double orc_integrate(int nlam, const double *nu, const double *spec) {
  double L = 0.0;
  for (int i = 0; i < nlam - 1; ++i) L = L + (fabs(nu[i] - nu[i + 1]) * 0.5) * (spec[i] + spec[i + 1]);
  return L;
}

/* T^4 of an integer temperature step.  The reference evaluates real(i)**4 in
 * single precision; the plain FP64 path uses double. */
static double t4(int i) {
  double d = (double)i;
  double d2 = d * d;
  return d2 * d2;
}

/* 1: the interpolations below form real(i)**4 in single precision as the
 * reference does (Radiation.f:551, 584, 698), (x x)(x x) with x = real(i),
 * their difference a single-precision subtraction widened to double */
static int t4_single = 0;
void orc_set_t4_single(int on) { t4_single = on != 0; }

static float t4f(int i) {
  const float x = (float)i;
  const float x2 = x * x;
  return x2 * x2;
}

static double t4_interp(int i, int j, double num, double den) {
  if (t4_single) {
    const float a = t4f(i), d = t4f(j) - t4f(i);
    return (double)a + ((double)d * num) / den;
  }
  return t4(i) + ((t4(j) - t4(i)) * num) / den;
}

/* (x)^(1/4) as sqrt(sqrt(x)): within 1 ulp of pow(x, 0.25), deterministic on
 * host and device */
static double qroot(double x) { return sqrt(sqrt(x)); }

static double computeE(const double *kp, int iT) {
  if (iT > ORC_TMAX) iT = ORC_TMAX;
  if (iT < 1) iT = 1;
  return kp[iT];
}

double orc_determine_t(const double *kp, double E1, double Tcur) {
  int iTmin = 1, iTmax = ORC_TMAX;
  int iT = (int)(Tcur / 1.0);
  if (iT < 1) iT = 1;
  if (iT > ORC_TMAX - 1) iT = ORC_TMAX - 1;
  double E = computeE(kp, iT);
  double Emax = computeE(kp, iTmax);
  double Emin = computeE(kp, 1);
  if (E1 != E1) return 3.0;
  if (E1 > Emax) return (double)(ORC_TMAX - 1);
  if (E1 < Emin) return 1.0;
  int iT0 = iT;
  int niter = 0;
  while (abs(iTmax - iTmin) > 1 && niter <= ORC_TMAX) {
    niter++;
    iT = (int)(qroot(E1 / E) * (double)iT);
    if (iT == iT0) {
      if (E1 < E) iT = iT0 - 1;
      if (E1 > E) iT = iT0 + 1;
    }
    for (;;) {
      if (iT <= iTmin) {
        iT = iTmin + 1;
        continue;
      }
      if (iT >= iTmax) {
        iT = iTmax - 1;
        continue;
      }
      break;
    }
    E = computeE(kp, iT);
    if (E >= E1) {
      iTmax = iT;
      Emax = E;
    }
    if (E <= E1) {
      iTmin = iT;
      Emin = E;
    }
    iT0 = iT;
  }
  if (iTmin == iTmax) return (double)iTmin;
  return qroot(t4_interp(iTmin, iTmax, E1 - Emin, Emax - Emin));
}

double orc_increase_t(const double *kp, double E1, double Tcur) {
  int j = (int)(Tcur / 1.0);
  if (j > ORC_TMAX) j = ORC_TMAX;
  if (j < 1) j = 1; /* computeE clamps its (by-reference) argument */
  double kp0 = kp[j];
  for (int i = j; i <= ORC_TMAX - 1; ++i) {
    double kp1 = kp[i + 1];
    if (kp0 <= E1 && kp1 >= E1)
      return qroot(t4_interp(i, i + 1, E1 - kp0, kp1 - kp0));
    kp0 = kp1;
  }
  return orc_determine_t(kp, E1, Tcur);
}

double orc_ran1(int32_t *idum, int32_t *iv, int32_t *iy) {
  const int32_t IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836, NTAB = 32;
  const int32_t NDIV = 1 + (IM - 1) / NTAB;
  const double AM = (double)(1.0f / (float)IM); /* single-precision constant */
  const double RNMX = 1.0 - (double)1.2e-7f;
  int32_t k;
  if (*idum <= 0 || *iy == 0) {
    *idum = (-*idum > 1) ? -*idum : 1;
    for (int j = NTAB + 8; j >= 1; --j) {
      k = *idum / IQ;
      *idum = IA * (*idum - k * IQ) - IR * k;
      if (*idum < 0) *idum += IM;
      if (j <= NTAB) iv[j - 1] = *idum;
    }
    *iy = iv[0];
  }
  k = *idum / IQ;
  *idum = IA * (*idum - k * IQ) - IR * k;
  if (*idum < 0) *idum += IM;
  int j = 1 + *iy / NDIV;
  *iy = iv[j - 1];
  iv[j - 1] = *idum;
  double r = AM * (double)*iy;
  return r < RNMX ? r : RNMX;
}

/* ---------------------------------------------------------------------
 * Per-component and per-cell tables read by the packet loop.
 * A "component" q is one (grain, opacity-set) pair of the reference;
 * comp_w[c*ncomp+q] = w(ii)*wopac(ii,iopac) of cell c.
 * --------------------------------------------------------------------- */

/* Planck means Kp(q,iT) = integrate(BB(:,iT)*Kabs_q), Init.f:3783-3790 */
void orc_kp_table(int nlam, const double *nu, const double *BB, int ncomp, const double *Kabs_comp,
                  double *Kp) {
  double *spec = (double *)malloc(sizeof(double) * (size_t)nlam);
  for (int q = 0; q < ncomp; ++q)
    for (int j = 0; j <= ORC_TMAX; ++j) {
      for (int l = 0; l < nlam; ++l) spec[l] = BB[(size_t)l * (ORC_TMAX + 1) + j] * Kabs_comp[(size_t)q * nlam + l];
      Kp[(size_t)q * (ORC_TMAX + 1) + j] = orc_integrate(nlam, nu, spec);
    }
  free(spec);
}

/* KabsTot/KscaTot per cell (MCRadiation.f:199-236) and the cell's Planck
 * mean table used by computeE (Radiation.f:611-627) */
void orc_cell_tables(int ncell, int ncomp, int nlam, const double *comp_w, const double *Kabs_comp,
                     const double *Ksca_comp, const double *Kp_comp, double *KabsTot, double *KscaTot,
                     double *KpCell) {
  /* cells are independent; each keeps the reference's summation order */
#pragma omp parallel for schedule(static)
  for (int c = 0; c < ncell; ++c) {
    const double *w = comp_w + (size_t)c * ncomp;
    for (int l = 0; l < nlam; ++l) {
      double a = 0.0, s = 0.0;
      for (int q = 0; q < ncomp; ++q) {
        a = a + Kabs_comp[(size_t)q * nlam + l] * w[q];
        s = s + Ksca_comp[(size_t)q * nlam + l] * w[q];
      }
      KabsTot[(size_t)c * nlam + l] = a;
      KscaTot[(size_t)c * nlam + l] = s;
    }
    for (int j = 0; j <= ORC_TMAX; ++j) {
      double e = 0.0;
      for (int q = 0; q < ncomp; ++q) e = e + Kp_comp[(size_t)q * (ORC_TMAX + 1) + j] * w[q];
      KpCell[(size_t)c * (ORC_TMAX + 1) + j] = e;
    }
  }
}

/* IF11, IF12 of every (component, wavelength) matrix, Init.f:3766-3776 */
void orc_if_table(int nmat, const double *F, const double *sinthet, double *IF) {
  const double pi = 3.14159265358979323846;
  for (int k = 0; k < nmat; ++k) {
    const double *F11 = F + (size_t)k * 1080, *F12 = F11 + 180;
    double a = 0.0, b = 0.0;
    for (int j = 0; j < 180; ++j) {
      a = a + ((pi * sinthet[j]) * F11[j]) / 180.0;
      b = b + ((pi * sinthet[j]) * F12[j]) / 180.0;
    }
    IF[2 * k] = a;
    IF[2 * k + 1] = b;
  }
}

/* asymmetry parameter g of every matrix, Init.f:4038-4050 */
void orc_g_table(int nmat, const double *F, double *g) {
  const double pi = 3.14159265358979323846;
  for (int k = 0; k < nmat; ++k) {
    const double *F11 = F + (size_t)k * 1080;
    double gg = 0.0, tot = 0.0;
    for (int ia = 1; ia <= 180; ++ia) {
      double s = sin(pi * ((double)ia - 0.5) / 180.0);
      gg = gg + (F11[ia - 1] * cos(pi * ((double)ia - 0.5) / 180.0)) * s;
      tot = tot + F11[ia - 1] * s;
    }
    g[k] = gg / tot;
  }
}

/* first-passage table of the random walk, RandomWalk.f:152-171 */
void orc_rw_table(double *y, double *phi) {
  const int NY = 1000;
  y[0] = 1.0;
  phi[0] = 1.0;
  for (int i = 2; i <= NY; ++i) {
    double yy = (double)(NY - i + 1) / (double)(NY - 1) * 0.75;
    y[i - 1] = yy;
    double p = 0.0;
    for (int n = 1; n <= 1000; ++n) {
      /* y^(n^2) by repeated squaring of the exponent bits */
      long long e = (long long)n * n;
      double base = yy, acc = 1.0;
      while (e) {
        if (e & 1) acc *= base;
        base *= base;
        e >>= 1;
      }
      p = p + ((n + 1) % 2 == 0 ? 1.0 : -1.0) * acc;
    }
    phi[i - 1] = p * 2.0;
  }
}

/* DiffCoeffCell (Dtable.f:97-182) for one cell and all iT in [1, TMAX-1]:
 * KDext(iT) = int dB / int dB/(Kext - g^2 Ksca), KDabs(iT) = int dB Kabs / int dB */
void orc_diffcoeff_cell(int nlam, const double *nu, const double *BB, const double *KabsTot,
                        const double *KscaTot, const double *gcell, int scattering, double *KDext,
                        double *KDabs) {
  double *spec = (double *)malloc(sizeof(double) * (size_t)nlam);
  double *dBB = (double *)malloc(sizeof(double) * (size_t)nlam);
  const int TT = ORC_TMAX + 1;
  KDext[0] = KDabs[0] = 0.0;
  KDext[ORC_TMAX] = KDabs[ORC_TMAX] = 0.0;
  for (int iT = 1; iT <= ORC_TMAX - 1; ++iT) {
    for (int l = 0; l < nlam; ++l) {
      dBB[l] = BB[(size_t)l * TT + iT + 1] - BB[(size_t)l * TT + iT];
      double g = scattering ? gcell[l] : 0.0;
      double Kext = KabsTot[l] + KscaTot[l];
      spec[l] = dBB[l] / (Kext - (g * g) * KscaTot[l]);
    }
    double int1 = orc_integrate(nlam, nu, spec);
    double int2 = orc_integrate(nlam, nu, dBB);
    KDext[iT] = int2 / int1;
    for (int l = 0; l < nlam; ++l) spec[l] = dBB[l] * (KabsTot[l] - 0.0);
    int1 = orc_integrate(nlam, nu, spec);
    KDabs[iT] = int1 / int2;
  }
  free(spec);
  free(dBB);
}

/* per-cell mean asymmetry g(l) = sum_q g_q Ksca_q w_q / KscaTot (Dtable.f:130-150) */
void orc_cell_g(int ncomp, int nlam, const double *w, const double *g_comp, const double *Ksca_comp,
                const double *KscaTot, double *gcell) {
  for (int l = 0; l < nlam; ++l) {
    double g = 0.0;
    for (int q = 0; q < ncomp; ++q) g = g + (g_comp[(size_t)q * nlam + l] * Ksca_comp[(size_t)q * nlam + l]) * w[q];
    gcell[l] = g / KscaTot[l];
  }
}

/* constant angle tables: sin(pi (i-1/2)/180) for the scattering-angle bins
 * (Radiation.f:449, Init.f:3771) and cos/sin(2 phi) with phi = pi (i-1)/179.5
 * (Init.f:3777-3781) */
void orc_const_tables(double *sinthet, double *cos2phi, double *sin2phi) {
  const double pi = 3.14159265358979323846;
  for (int i = 1; i <= 180; ++i) sinthet[i - 1] = sin((pi * ((double)i - 0.5)) / 180.0);
  for (int i = 0; i <= 360; ++i) {
    double phi = (pi * (double)(i - 1)) / 179.5;
    cos2phi[i] = cos(2.0 * phi);
    sin2phi[i] = sin(2.0 * phi);
  }
}
