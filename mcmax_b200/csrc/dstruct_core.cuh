/*
 * dstruct_core.cuh -- the vertical structure of the disk (DiskStructure,
 * DiskStructure.f:85-468): per ring and per species (gas and each grain) the
 * density profile along theta from hydrostatic equilibrium in the current
 * temperatures, renormalised to the species' mass in the ring, then the
 * cells' densities and abundances rebuilt from the profiles
 * (DiskStructure.f:392-449, CheckMinimumDensity DiskStructure.f:2966,
 * CheckCells DiskStructure.f:2659).
 *
 * Built: 'DISK' scale-height species, gas included, zones with a fixed
 * structure (the analytic profile of DiskStructure.f:360-386, wedges too),
 * per-ring scale factors and per-grain settling factors as inputs, and the
 * other scale-height types of DiskStructure.f:248-344 (ZODI, HALO, LOBE,
 * JET, SHELL, CYLI, CAVITY, WEDGE, and an unknown type that keeps the
 * grain's current densities).  Those closed-form profiles are formed on the
 * host with the C library's functions (ds_shape_profile) and only
 * renormalised on the device.  Not built: radiation pressure (beta = 0),
 * mpstr, scset settling, gaps, halo, radial structure iterations.
 *
 * Shared by the library (dstruct.cu: one thread per column, one per cell)
 * and the host replay of the tests.  Every a*b+c is rounded twice (the unit
 * is built with --fmad=false, the replay with -ffp-contract=off) and exp,
 * log and the step-size powers come from detmath.h, so the two agree bit for
 * bit.  The ODE integrator is odeint/rkqs/rkck of Subroutines.f:1933-2090
 * (Cash-Karp Runge-Kutta with adaptive steps, as published in Numerical
 * Recipes), with its constants at the values the reference gives them:
 * single-precision literals widened to double.
 */
#ifndef MCMAX_DSTRUCT_CORE_CUH
#define MCMAX_DSTRUCT_CORE_CUH

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "detmath.h"

#ifdef __CUDACC__
#define DS_HD __host__ __device__ inline
#else
#define DS_HD static inline
#endif

#define DS_AU ((double)1.49598e13f)                      /* Modules.f:8 */
#define DS_PI 3.14159265358979323846
#define DS_MU (0x1.2666660000000p+1 * 1.67262158e-24)   /* DiskStructure.f:475: 2.3 as a float */
#define DS_G 6.67300e-8                                  /* DiskStructure.f:477 */
#define DS_KB 1.3806503e-16                              /* Modules.f:11 */

/* scale-height types of a grain (Grain(ii)%shtype, Init.f:920-926) */
enum {
  DS_SH_DISK = 0,   /* hydrostatic equilibrium */
  DS_SH_ZODI = 1,   /* zodiacal cosine model */
  DS_SH_HALO = 2,   /* constant, a wedge when the grain's factor is negative */
  DS_SH_LOBE = 3,   /* Gaussian in theta, width scale degrees */
  DS_SH_JET = 4,    /* Gaussian in theta, width growing with radius */
  DS_SH_SHELL = 5,  /* 1 + factor sin^3 theta */
  DS_SH_CYLI = 6,   /* cylinder of height scale AU */
  DS_SH_CAVITY = 7, /* outside a paraboloidal cavity */
  DS_SH_WEDGE = 8,  /* theta above (or below) scale degrees */
  DS_SH_KEEP = 9,   /* an unknown type: the grain's densities as they are */
  DS_SH_NTYPES = 10
};

/* one ODE segment: d ln(rho)/dz between z1 (cell j+1) and z2 (cell j), the
 * temperature linear in z between the two cell temperatures (derivs,
 * DiskStructure.f:469-491, without radiation pressure) */
struct DsSeg {
  double z1, z2, T1, T2, dlnT; /* the segment and its end temperatures */
  double A, scale2kb, R3;      /* mu G Mstar, scale^2 kb, R_av^3 */
};

DS_HD double ds_derivs(const DsSeg &s, double x) {
  const double T = s.T1 + ((s.T2 - s.T1) * (x - s.z1)) / (s.z2 - s.z1);
  return -(s.A * x) / ((s.scale2kb * T) * s.R3) - s.dlnT; /* (1 + beta) = 1 */
}

DS_HD double ds_pow(double x, double y) { return dm_exp(y * dm_log(x)); }

/* rkck + rkqs (Subroutines.f:1997-2090).  The right-hand side does not
 * depend on y, so the intermediate y values of the stages are not formed. */
DS_HD void ds_rkqs(const DsSeg &s, double *y, double dydx, double *x, double htry, double eps, double yscal,
                   double *hdid, double *hnext) {
  /* the reference's single-precision literals and quotients (0.9, -.2,
   * 1.89e-4, .3, .6, .875, 37./378., 250./621., 125./594., 512./1771.,
   * 2825./27648., 18575./48384., 13525./55296., -277./14336.) rounded to
   * float and widened, written out exactly */
  const double SAFETY = 0x1.cccccc0000000p-1, PGROW = -0x1.99999a0000000p-3, PSHRNK = -0.25,
               ERRCON = 0x1.8c5c9a0000000p-13;
  const double A3 = 0x1.3333340000000p-2, A4 = 0x1.3333340000000p-1, A5 = 1.0, A6 = 0.875;
  const double C1 = 0x1.90ee640000000p-4, C3 = 0x1.9c3d020000000p-2, C4 = 0x1.aef9f80000000p-3,
               C6 = 0x1.280a680000000p-2;
  const double DC1 = C1 - 0x1.a284be0000000p-4, DC3 = C3 - 0x1.891f280000000p-2, DC4 = C4 - 0x1.f4ed0a0000000p-3,
               DC5 = -0x1.3c924a0000000p-6, DC6 = C6 - 0.25;
  double h = htry;
  for (int guard = 0; guard < 200; ++guard) {
    const double ak3 = ds_derivs(s, *x + A3 * h), ak4 = ds_derivs(s, *x + A4 * h);
    const double ak5 = ds_derivs(s, *x + A5 * h), ak6 = ds_derivs(s, *x + A6 * h);
    const double ytemp = *y + h * (((C1 * dydx + C3 * ak3) + C4 * ak4) + C6 * ak6);
    const double yerr = h * ((((DC1 * dydx + DC3 * ak3) + DC4 * ak4) + DC5 * ak5) + DC6 * ak6);
    double errmax = fabs(yerr / yscal);
    if (!(errmax > 0.0)) errmax = 0.0;
    errmax = errmax / eps;
    if (errmax > 1.0) {
      const double htemp = (SAFETY * h) * ds_pow(errmax, PSHRNK);
      h = copysign(fmax(fabs(htemp), 0x1.99999a0000000p-4 * fabs(h)), h); /* 0.1 as a float */
      continue;
    }
    *hnext = errmax > ERRCON ? (SAFETY * h) * ds_pow(errmax, PGROW) : 5.0 * h;
    *hdid = h;
    *x = *x + h;
    *y = ytemp;
    return;
  }
  /* the reference retries without bound; each retry shrinks h by a factor
   * between 0.1 and 0.9, so 200 retries take it below 1e-9 of the first
   * try and this is not reached for finite input */
  *hdid = h;
  *hnext = h;
  *x = *x + h;
}

/* odeint (Subroutines.f:1933-1994) with hmin = 0 and no stored path */
DS_HD double ds_odeint(const DsSeg &s, double ystart, double eps, double h1) {
  const double x1 = s.z1, x2 = s.z2, TINY = 1.e-150;
  double x = x1, y = ystart;
  double h = copysign(fabs(h1), x2 - x1);
  for (int nstp = 1; nstp <= 10000; ++nstp) {
    const double dydx = ds_derivs(s, x);
    const double yscal = (fabs(y) + fabs(h * dydx)) + TINY;
    if (((x + h) - x2) * ((x + h) - x1) > 0.0) h = x2 - x;
    double hdid, hnext;
    ds_rkqs(s, &y, dydx, &x, h, eps, yscal, &hdid, &hnext);
    if ((x - x2) * (x2 - x1) >= 0.0) return y;
    h = hnext;
  }
  return y;
}

/* one (ring, species) column: the log-density profile along j = 1..nc (nc =
 * nTheta-1, j = nc at the midplane), then exp, renormalised to mass M0 and
 * floored at 1e-50 (DiskStructure.f:200-390).
 *   Trow    the ring's temperatures, Trow[j-1] for cell j
 *   Vrow    the ring's cell volumes
 *   z, st, ct, cot  per cell j-1: R_av cos(theta_av), sin, cos, 1/tan of theta_av
 *   fix     < 0: hydrostatic; else the fixed zone's (sh, rsh, shpow, denspow)
 *   rho     out, nc values */
struct DsColumn {
  int fix;          /* index of a fixed-structure zone containing the ring, or -1 */
  long long pre;    /* offset of a closed-form log profile formed on the host, or -1 */
  double scale;     /* scale-height factor of the species in the ring */
  double M0;        /* the species' mass in the ring */
  double sh, rsh, shpow, denspow; /* the fixed zone's profile */
};

DS_HD void ds_column(const DsColumn &col, int nc, double R_av, double Mstar, const double *Trow, const double *Vrow,
                     const double *z, const double *st, const double *ct, const double *cot,
                     const double *theta_av, const double *pre, double *rho) {
  if (pre) {
    for (int j = 0; j < nc; ++j) rho[j] = pre[j];
  } else if (col.fix < 0) {
    rho[nc - 1] = 0.0;
    if (col.scale > 0.0) {
      DsSeg s;
      s.A = (DS_MU * DS_G) * Mstar;
      s.scale2kb = (col.scale * col.scale) * DS_KB;
      s.R3 = (R_av * R_av) * R_av;
      for (int j = nc - 1; j >= 1; --j) { /* cell j from cell j+1 */
        s.z1 = z[j];
        s.z2 = z[j - 1];
        s.T1 = Trow[j];
        s.T2 = Trow[j - 1];
        s.dlnT = (dm_log(s.T1) - dm_log(s.T2)) / (s.z1 - s.z2);
        const double h1 = fabs(s.z2 - s.z1) * 1e-6;
        rho[j - 1] = ds_odeint(s, rho[j], 1e-6, h1);
      }
    } else { /* wedge */
      for (int j = nc - 1; j >= 1; --j) rho[j - 1] = (cot[j - 1] < -col.scale) ? 0.0 : -60.0;
    }
  } else if (col.sh < 0.0) { /* wedge zone */
    rho[nc - 1] = 0.0;
    for (int j = 1; j <= nc - 1; ++j) rho[j - 1] = ((180.0 * theta_av[j - 1]) / DS_PI > -col.sh) ? 0.0 : -60.0;
  } else {
    for (int j = 1; j <= nc; ++j) {
      const double rr = (R_av * st[j - 1]) / DS_AU, zz = (R_av * ct[j - 1]) / DS_AU;
      const double hr = (col.scale * col.sh) * ds_pow(rr / col.rsh, col.shpow);
      const double f1 = ds_pow(rr, -col.denspow);
      double f2 = -((zz / hr) * (zz / hr));
      if (j == nc) f2 = 0.0;
      rho[j - 1] = dm_log(f1 / hr) + f2;
    }
  }
  double M1 = 0.0;
  for (int j = 0; j < nc; ++j) M1 = M1 + dm_exp(rho[j]) * Vrow[j];
  for (int j = 0; j < nc; ++j) {
    double r = (dm_exp(rho[j]) * col.M0) / M1;
    if (r < 1e-50) r = 1e-50;
    rho[j] = r;
  }
}

/* rebuild one cell (i >= 1) from the profiles (DiskStructure.f:392-449 and
 * CheckMinimumDensity): rho[k*stride] is the new density of species k (0
 * gas, 1..ng grains).  dens, dens0, gasdens, w[ng], w0[ng] in/out.  w holds
 * the gas fractions, then the new abundances, so no scratch is needed. */
DS_HD void ds_cell(int ng, const double *rho, size_t stride, double *dens, double *dens0, double *gasdens, double *w,
                   double *w0) {
  for (int k = 0; k < ng; ++k) {
    double g;
    if (w0[k] >= 1e-100)
      g = 1.0 - (*dens * w[k]) / (*dens0 * w0[k]);
    else
      g = 0.0;
    if (g < 0.0) g = 0.0;
    if (g > 1.0) g = 1.0;
    if (g != g) g = 0.0;
    w[k] = g;
  }
  *gasdens = rho[0];
  double d0 = 0.0;
  for (int k = 0; k < ng; ++k) d0 = d0 + rho[(size_t)(1 + k) * stride];
  *dens0 = d0;
  if (d0 > 1e-50)
    for (int k = 0; k < ng; ++k) w0[k] = rho[(size_t)(1 + k) * stride] / d0;
  double t = 0.0;
  for (int k = 0; k < ng; ++k) t = t + w0[k];
  for (int k = 0; k < ng; ++k) {
    w0[k] = w0[k] / t;
    w[k] = w0[k] * (1.0 - w[k]);
  }
  t = 0.0;
  for (int k = 0; k < ng; ++k) t = t + w[k];
  if (t > 1e-50)
    for (int k = 0; k < ng; ++k) w[k] = w[k] / t;
  else
    for (int k = 0; k < ng; ++k) w[k] = w0[k];
  *dens = *dens0 * t;
  /* CheckMinimumDensity (DiskStructure.f:2966-3010) */
  if (*dens0 <= 1e-50) *dens0 = 1e-50;
  if (*dens <= 1e-50) *dens = 1e-50;
  if (*gasdens <= 1e-50) *gasdens = 1e-50;
  const double dold = *dens;
  for (int k = 0; k < ng; ++k) {
    double m = dold * w[k];
    if (m < 1e-50) m = 1e-50;
    if (m > *dens0 * w0[k]) m = *dens0 * w0[k];
    w[k] = m;
  }
  double d = 0.0;
  for (int k = 0; k < ng; ++k) d = d + w[k];
  *dens = d;
  if (*dens <= 1e-50) {
    *dens = 1e-50;
    for (int k = 0; k < ng; ++k) w[k] = w0[k];
  } else {
    for (int k = 0; k < ng; ++k) w[k] = w[k] / *dens;
  }
}

/* CheckCells (DiskStructure.f:2659-2697) for one cell */
DS_HD void ds_check_cell(int ng, double *dens, double dens0, double *w, const double *w0) {
  bool rescale = false;
  for (int k = 0; k < ng; ++k)
    if (*dens * w[k] > dens0 * w0[k]) rescale = true;
  if (!rescale) return;
  const double dold = *dens;
  double d = 0.0;
  for (int k = 0; k < ng; ++k) {
    double m = dold * w[k];
    if (m > dens0 * w0[k]) m = dens0 * w0[k];
    w[k] = m;
    d = d + m;
  }
  *dens = d;
  if (d > 1e-50) {
    for (int k = 0; k < ng; ++k) w[k] = w[k] / d;
  } else {
    *dens = 1e-50;
    for (int k = 0; k < ng; ++k) w[k] = w0[k];
  }
}

/* ------------------------------------------------------------ host logic */

struct DsZone {
  double rin, rout;         /* AU */
  double sh, rsh, shpow, denspow;
  int fix_struct;
};

struct DsGrid {
  int nr, nt, ng;           /* D%nR, D%nTheta, grains */
  const double *R;          /* nr+1, AU */
  const double *Theta;      /* nt, cos theta edges */
  const double *V;          /* ncell */
  double Mstar;             /* g */
  int nzones;
  const DsZone *zones;
  const double *shscale;    /* nr, or NULL (1) */
  const double *gscale;     /* ng*nr settling factor of each grain per ring, or NULL (1) */
  const int *shtype;        /* ng scale-height types (DS_SH_*), or NULL (all DS_SH_DISK) */
};

/* per-ring and per-theta geometry, computed on the host */
struct DsTables {
  std::vector<double> R_av, z, st, ct, cot, theta_av, thet; /* R_av[nr]; z[nr*nc]; the rest [nc] */
};

static inline void ds_tables(const DsGrid &g, DsTables *t) {
  const int nR = g.nr, nc = g.nt - 1;
  t->R_av.assign(nR, 0.0);
  t->z.assign((size_t)nR * nc, 0.0);
  t->st.assign(nc, 0.0);
  t->ct.assign(nc, 0.0);
  t->cot.assign(nc, 0.0);
  t->theta_av.assign(nc, 0.0);
  t->thet.assign(nc, 0.0);
  for (int i = 0; i < nR; ++i) t->R_av[i] = DS_AU * pow(10.0, (log10(g.R[i]) + log10(g.R[i + 1])) / 2.0);
  for (int j = 1; j <= nc; ++j) {
    const double th = acos((g.Theta[j - 1] + g.Theta[j]) / 2.0);
    t->theta_av[j - 1] = th;
    t->st[j - 1] = sin(th);
    t->ct[j - 1] = cos(th);
    t->cot[j - 1] = 1.0 / tan(th);
    t->thet[j - 1] = acos(g.Theta[j - 1]); /* D%thet(j), the cell's polar edge */
  }
  for (int i = 0; i < nR; ++i)
    for (int j = 0; j < nc; ++j) t->z[(size_t)i * nc + j] = t->R_av[i] * t->ct[j];
}

/* the column set-up of DiskStructure.f:150-198 for ring i (1..nR-1) and
 * species k (0 gas, 1..ng grains) */
static inline DsColumn ds_setup_column(const DsGrid &g, const DsTables &t, int i, int k, const double *dens,
                                       const double *dens0, const double *gasdens, const double *w, const double *w0) {
  const int nc = g.nt - 1, ng = g.ng;
  DsColumn col;
  const double ring = g.shscale ? g.shscale[i] : 1.0;
  col.scale = 1.0 * ring;
  if (k > 0 && g.gscale) col.scale = ring * g.gscale[(size_t)(k - 1) * g.nr + i];
  double M0 = 0.0;
  for (int j = 0; j < nc; ++j) {
    const size_t c = (size_t)i * nc + j;
    if (k > 0)
      M0 = M0 + (dens0[c] * g.V[c]) * w0[c * ng + (k - 1)];
    else
      M0 = M0 + gasdens[c] * g.V[c];
  }
  col.M0 = M0;
  int fix = -1;
  const double Rav = t.R_av[i];
  for (int iz = 0; iz < g.nzones; ++iz) {
    const DsZone &zn = g.zones[iz];
    if (Rav > zn.rin * DS_AU && Rav < zn.rout * DS_AU && zn.fix_struct) fix = iz;
  }
  if (k == 0)
    for (int iz = 0; iz < g.nzones; ++iz) {
      const DsZone &zn = g.zones[iz];
      if (Rav > zn.rin * DS_AU && Rav < zn.rout * DS_AU && !zn.fix_struct) fix = -1;
    }
  col.fix = fix;
  col.pre = -1;
  col.sh = col.rsh = col.shpow = col.denspow = 0.0;
  if (fix >= 0) {
    col.sh = g.zones[fix].sh;
    col.rsh = g.zones[fix].rsh;
    col.shpow = g.zones[fix].shpow;
    col.denspow = g.zones[fix].denspow;
  }
  return col;
}

/* the closed-form log-density profiles of the scale-height types other than
 * DISK (DiskStructure.f:248-344) for grain k (1..ng) in ring i, formed on
 * the host with the C library's functions, in the reference's operation
 * order.  scale: the column's factor (ring times grain); gsh: the grain's own
 * factor Grain(ii)%shscale(i), which HALO and SHELL read; dens, w: the cell
 * arrays as they are (the unknown type keeps log(dens w)). */
static inline void ds_shape_profile(const DsGrid &g, const DsTables &t, int i, int k, int type, double scale,
                                    const double *dens, const double *w, double *rho) {
  const int nc = g.nt - 1, ng = g.ng;
  const double gsh = g.gscale ? g.gscale[(size_t)(k - 1) * g.nr + i] : 1.0;
  const double *z = &t.z[(size_t)i * nc];
  const double Rav = t.R_av[i], Rout = t.R_av[g.nr - 1];
  for (int j = 0; j < nc; ++j) {
    const double th = t.theta_av[j], deg = (180.0 * th) / DS_PI;
    double r = 0.0;
    switch (type) {
      case DS_SH_ZODI: /* cosine model (Rittich 1986), DiskStructure.f:249-255 */
        r = log(0.15 + (double)0.85f * pow(cos(DS_PI / 2.0 - th), 28.0));
        break;
      case DS_SH_HALO:
        r = (gsh < 0.0 && DS_PI / 2.0 - th > -gsh) ? -60.0 : 0.0;
        break;
      case DS_SH_LOBE: {
        const double q = deg / scale;
        r = log10(exp(-(q * q)));
        break;
      }
      case DS_SH_JET: {
        const double q = ((t.thet[j] * 180.0) / DS_PI) / (scale * (Rav / Rout));
        r = -(q * q);
        break;
      }
      case DS_SH_SHELL:
        r = log(1.0 + gsh * pow(sin(th), 3.0));
        break;
      case DS_SH_CYLI:
        r = (j == nc - 1 || z[j] / DS_AU < scale) ? 0.0 : -60.0;
        break;
      case DS_SH_CAVITY: {
        const double rc = (Rav * t.st[j]) / DS_AU;
        r = (j == nc - 1) ? 0.0 : (j == 0) ? -60.0 : (z[j] / DS_AU < (rc * rc) * scale) ? 0.0 : -60.0;
        break;
      }
      case DS_SH_WEDGE:
        r = scale > 0.0 ? (deg > scale ? 0.0 : -60.0) : (deg < -scale ? 0.0 : -60.0);
        break;
      default: { /* DS_SH_KEEP */
        const size_t c = (size_t)i * nc + j;
        const double v = dens[c] * w[c * ng + (k - 1)];
        r = v > 1e-60 ? log(v) : -60.0;
      }
    }
    rho[j] = r;
  }
}

/* Backend: columns(g, t, Temp, ncol, cols, ring, prof, rho[ncol*nc]) runs
 * ds_column per column (prof: the host-formed profiles the columns' pre
 * offsets point into), cells(g, rho, dens, dens0, gasdens, w, w0) runs
 * ds_cell per cell of rings 1..nR-1 and then ds_check_cell per cell of
 * rings 0..nR-1; each returns false on an execution error.  Cell arrays:
 * dens, dens0, gasdens (ncell), w, w0 (ncell*ng), all in/out. */
template <class Backend>
bool ds_disk_structure(const DsGrid &g, Backend &be, const double *Temp, double *dens, double *dens0,
                       double *gasdens, double *w, double *w0) {
  const int nR = g.nr, nc = g.nt - 1, ns = g.ng + 1;
  if (nR < 2 || nc < 2 || g.ng < 1) return true;
  DsTables t;
  ds_tables(g, &t);
  const int ncol = (nR - 1) * ns;
  std::vector<DsColumn> cols(ncol);
  std::vector<int> ring(ncol);
  std::vector<double> prof;
  for (int i = 1; i < nR; ++i)
    for (int k = 0; k < ns; ++k) {
      const int q = (i - 1) * ns + k;
      cols[q] = ds_setup_column(g, t, i, k, dens, dens0, gasdens, w, w0);
      ring[q] = i;
      const int type = (k > 0 && g.shtype) ? g.shtype[k - 1] : DS_SH_DISK;
      if (cols[q].fix < 0 && type != DS_SH_DISK) {
        cols[q].pre = (long long)prof.size();
        prof.resize(prof.size() + nc);
        ds_shape_profile(g, t, i, k, type, cols[q].scale, dens, w, &prof[(size_t)cols[q].pre]);
      }
    }
  std::vector<double> rho((size_t)ncol * nc);
  if (!be.columns(g, t, Temp, ncol, cols.data(), ring.data(), prof, rho.data())) return false;
  return be.cells(g, rho.data(), dens, dens0, gasdens, w, w0);
}

/* serial loops of the two steps (host backend and replay) */
static inline void ds_columns_host(const DsGrid &g, const DsTables &t, const double *Temp, int ncol,
                                   const DsColumn *cols, const int *ring, const std::vector<double> &prof,
                                   double *rho) {
  const int nc = g.nt - 1;
  for (int q = 0; q < ncol; ++q) {
    const int i = ring[q];
    ds_column(cols[q], nc, t.R_av[i], g.Mstar, Temp + (size_t)i * nc, g.V + (size_t)i * nc, &t.z[(size_t)i * nc],
              t.st.data(), t.ct.data(), t.cot.data(), t.theta_av.data(),
              cols[q].pre >= 0 ? &prof[(size_t)cols[q].pre] : nullptr, rho + (size_t)q * nc);
  }
}

static inline void ds_cells_host(const DsGrid &g, const double *rho, double *dens, double *dens0, double *gasdens,
                                 double *w, double *w0) {
  const int nR = g.nr, nc = g.nt - 1, ng = g.ng, ns = ng + 1;
  for (int i = 1; i < nR; ++i)
    for (int j = 0; j < nc; ++j) {
      const size_t c = (size_t)i * nc + j;
      ds_cell(ng, rho + (size_t)(i - 1) * ns * nc + j, nc, &dens[c], &dens0[c], &gasdens[c], &w[c * ng],
              &w0[c * ng]);
    }
  for (size_t c = 0; c < (size_t)nR * nc; ++c) ds_check_cell(ng, &dens[c], dens0[c], &w[c * ng], &w0[c * ng]);
}

#endif /* MCMAX_DSTRUCT_CORE_CUH */
