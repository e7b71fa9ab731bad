/*
 * surrogate_phase.h -- the Mueller matrix on ComputePart's 180 scattering-
 * angle bins from the opacity surrogate's Legendre moments (host code,
 * shared by mcg_compute_part_surrogate and the CPU test harness).
 *
 * Per wavelength the surrogate gives moments to order SURR_PH_L = 12 of F11
 * (chi_l, chi_0 = 1), F12 (beta_l), F33 (gamma_l) and F34 (delta_l), each a
 * sum over the bins mu_j = cos((j + 1/2) deg) with weights
 * w_j = sin((j + 1/2) deg), divided by F11's zeroth moment.  The series
 * sum_l (2l + 1) c_l P_l(mu_j) rebuilds each element.
 *
 * A truncated series of a strongly forward-peaked F11 rings and goes
 * negative.  Clipping it at zero and renormalising then changes the
 * asymmetry parameter: for the large grains of a disk at short wavelengths
 * g = 0.97 becomes 0.53.  The delta-M method (Wiscombe 1977, J. Atmos. Sci.
 * 34, 1408) avoids this.  It moves a forward fraction f into a delta
 * function, and the remainder's moments (chi_l - f) / (1 - f) fall to zero
 * at l = L.  That series stays close to non-negative, and the total keeps
 * the moments 0..L (g included) where it needs no clipping.  In the exact
 * forward direction a sphere has F33 = F11 and F12 = F34 = 0.  So the delta
 * goes into the first bin of F11 and of F33, with gamma_l -> (gamma_l - f) /
 * (1 - f), and F12 and F34 keep their moments (divided by 1 - f).
 * f = chi_L^2 / chi_{L-1}, the next moment of a Henyey-Greenstein function
 * with these two; it is capped at chi_L and at 0.99, and is 0 when either
 * moment is not positive.
 *
 * Constraints of any mixture of spheres, applied last: F11 >= 0 (clipped
 * before the normalisation), |F12| <= F11, F22 = F11, F44 = F33, and
 * F12^2 + F33^2 + F34^2 <= F11^2 (F33 and F34 scaled back where broken).
 */
#ifndef MCMAX_SURROGATE_PHASE_H
#define MCMAX_SURROGATE_PHASE_H

#include <math.h>

constexpr int SURR_PH_L = 12;   /* Legendre moments per element */
constexpr int SURR_PH_NA = 180; /* scattering-angle bins */

/* Legendre polynomials at the bin centres and the bins' weights */
struct SurrLegendre {
  double P[SURR_PH_L + 1][SURR_PH_NA];
  double w[SURR_PH_NA];
  double wsum = 0.0;
  SurrLegendre() {
    for (int j = 0; j < SURR_PH_NA; ++j) {
      const double th = 3.14159265358979323846 * ((double)j + 0.5) / (double)SURR_PH_NA;
      const double mu = cos(th);
      w[j] = sin(th);
      wsum += w[j];
      P[0][j] = 1.0;
      P[1][j] = mu;
      for (int l = 1; l < SURR_PH_L; ++l)
        P[l + 1][j] = ((2.0 * l + 1.0) * mu * P[l][j] - (double)l * P[l - 1][j]) / (l + 1);
    }
  }
};

/* the forward fraction of the delta-M method for F11's moments chi[0..L] */
inline double surr_deltam_fraction(const double *chi) {
  const double a = chi[SURR_PH_L - 1], b = chi[SURR_PH_L];
  if (!(a > 0.0) || !(b > 0.0)) return 0.0;
  double f = b * b / a;
  if (f > b) f = b;
  if (f > 0.99) f = 0.99;
  return f;
}

/* F[6][NA] (F11, F12, F22, F33, F34, F44) from the moments chi, beta, gam,
 * del [0..L]; deltam = 0 gives the plain clipped series */
inline void surr_phase_matrix(const SurrLegendre &T, const double *chi, const double *beta, const double *gam,
                              const double *del, int deltam, double *F) {
  constexpr int L = SURR_PH_L, NA = SURR_PH_NA;
  const double f = deltam ? surr_deltam_fraction(chi) : 0.0;
  const double rest = 1.0 - f;
  double cc[L + 1], bc[L + 1], gc[L + 1], dc[L + 1];
  for (int m = 0; m <= L; ++m) {
    cc[m] = (chi[m] - f) / rest;
    bc[m] = beta[m] / rest;
    gc[m] = (gam[m] - f) / rest;
    dc[m] = del[m] / rest;
  }
  double f11[NA], f12[NA], f33[NA], f34[NA], norm = 0.0;
  for (int j = 0; j < NA; ++j) {
    double a = 0.0, b = 0.0, g = 0.0, d = 0.0;
    for (int m = 0; m <= L; ++m) {
      a += (2.0 * m + 1.0) * cc[m] * T.P[m][j];
      b += (2.0 * m + 1.0) * bc[m] * T.P[m][j];
      g += (2.0 * m + 1.0) * gc[m] * T.P[m][j];
      d += (2.0 * m + 1.0) * dc[m] * T.P[m][j];
    }
    f11[j] = a > 0.0 ? a : 0.0;
    f12[j] = b;
    f33[j] = g;
    f34[j] = d;
    norm += f11[j] * T.w[j];
  }
  /* the remainder carries weight 1 - f of the bins' total, the delta f */
  const double c = norm > 0.0 ? T.wsum * rest / norm : 1.0;
  const double spike = f * T.wsum / T.w[0];
  for (int j = 0; j < NA; ++j) {
    double a = f11[j] * c, b = f12[j] * c, g = f33[j] * c, d = f34[j] * c;
    if (j == 0) {
      a += spike;
      g += spike;
    }
    if (b > a) b = a;
    if (b < -a) b = -a;
    const double room = a * a - b * b, gd = g * g + d * d;
    if (gd > room) {
      const double s = gd > 0.0 ? sqrt(room / gd) : 0.0;
      g *= s;
      d *= s;
    }
    F[0 * NA + j] = a;
    F[1 * NA + j] = b;
    F[2 * NA + j] = a;
    F[3 * NA + j] = g;
    F[4 * NA + j] = d;
    F[5 * NA + j] = g;
  }
}

#endif /* MCMAX_SURROGATE_PHASE_H */
