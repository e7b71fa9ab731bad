/*
 * oracle.h -- CPU restatement of the MCMax hot path, used ONLY as the test
 * reference for parity tests (tests/, the smoke check and bench.py's CPU baseline).  It is not
 * part of the product and the product never links it.
 *
 * Parity status: UNPINNED against the reference binary.  MCMax is Fortran,
 * there is no Fortran compiler, cfitsio or fftw3 in this image, and the
 * reference ships no tests or golden outputs.  The restatement follows the
 * reference source line by line (citations at each function) and is pinned by
 * known-answer checks (published Mie values, homogeneous-sphere limits of the
 * coated-sphere code, Bruggeman identities, energy conservation) in tests/.
 *
 * Precision: the "plain" path computes in FP64 throughout (the reference's
 * ComputePart passes REAL/COMPLEX single-precision values into its DOUBLE
 * PRECISION DMiLay; the plain path promotes those to double).  Elementary
 * functions on the per-sample path come from mcmax_b200/csrc/detmath.h (a
 * portable libm substitute) so the GPU result can be compared bit for bit.
 */
#ifndef MCMAX_ORACLE_H
#define MCMAX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NA 180          /* scattering-angle bins, ComputePart.f:41 */
#define ORC_TMAX 10000      /* Modules.f:5 */
#define ORC_NANGLE_SED 30   /* MCRadiation.f:20 */

/* ---------------- opacity stage (ComputePart.f) ---------------- */

/* Toon-Ackerman coated sphere, ComputePart.f:1256-1711.  Returns 0 or 1
 * (Err).  m1,m2,s21,d21 are [2][numang] (index k*numang + j). */
int orc_dmilay(double rcore, double rshell, double wvno, double shell_re, double shell_im,
               double core_re, double core_im, const double *mu, int numang, double *qext,
               double *qsca, double *qbs, double *gqsc, double *m1, double *m2, double *s21,
               double *d21);

/* Homogeneous-sphere Mie for one radius (MeerhoffMie, ComputePart.f:1883-1927
 * with mie/scatmat/fichid/anbn/pitau, :1932-3213).  F11..F34 have na entries,
 * index 0 = most forward bin.  Returns 0 or 1 when the term count would not
 * fit the recurrences. */
int orc_meerhoff_mie(double rad, double lam, double e1, double e2, double *csca, double *cext,
                     double *f11, double *f12, double *f33, double *f34, int na);

/* Bruggeman effective medium, ComputePart.f:1177-1212 */
void orc_blender(const double *e1, const double *e2, const double *abun, int nm, double *e1out,
                 double *e2out);

/* Gauss-Legendre nodes, ComputePart.f:1219-1249 */
void orc_gauleg2(double x1, double x2, double *x, double *w, int n);

/* One ComputePart call for already-read refractive indices
 * (standard='FILE' form, ComputePart.f:1-552).
 * in : nlam, lam[nlam] (micron), nm, e1[nm*nlam], e2[nm*nlam] (n and k of
 *      each material on the wavelength grid), frac[nm], rho[nm] (as read
 *      from the particle file, before the /rho conversion), amin, amax (micron),
 *      apow, fmax, blend, porosity, ns (sizes), nf (filling fractions),
 *      normalize_abun (<=0: none)
 * out: kabs,ksca,kext[nlam] (cm^2/g), F[nlam*6*180] (F11,F12,F22,F33,F34,F44
 *      blocks of 180 per wavelength), rho_av, mscale, rscale;
 *      counters[0] = number of DHS samples, counters[1] = Mie samples,
 *      counters[2] = DHS failures that fell back to Mie.
 * Returns 0, or -1 on invalid arguments. */
int orc_compute_part(int nlam, const double *lam, int nm, const double *e1, const double *e2,
                     const double *frac, const double *rho, double amin, double amax,
                     double apow, double fmax, int blend, double porosity, int ns, int nf,
                     double normalize_abun, double *kabs, double *ksca, double *kext, double *F,
                     double *rho_av, double *mscale, double *rscale, int64_t *counters);

/* ---------------- table builders (Init.f, Subroutines.f) ---------------- */

/* Planck B_nu(T, lam) with the quad-precision exponential, Subroutines.f:4-21 */
double orc_planck(double T, double lam);
/* BB[nlam*(TMAX+1)] row-major by wavelength: BB[l*(TMAX+1)+iT], Init.f:2616-2622 */
void orc_bb_table(int nlam, const double *lam, double *BB);
/* trapezoid over frequency, Radiation.f:1-18 */
double orc_integrate(int nlam, const double *nu, const double *spec);

/* ---------------- transport (MCRadiation.f, Radiation.f, RandomWalk.f) ---------------- */

typedef struct {
  /* grid: nr = D%nR (radial edges R[0..nr], R[0] = Rstar/AU), nt = D%nTheta
   * (cos-theta edges Theta[1..nt] stored at Theta[0..nt-1], Theta[0] = 1,
   * Theta[nt-1] = 0).  Cells: i = 0..nr-1, j = 1..nt-1, flattened as
   * c = i*(nt-1) + (j-1). */
  int nr, nt;
  const double *R;        /* nr+1 */
  const double *Theta;    /* nt   */
  const double *SinTheta; /* nt   */
  const double *dens;     /* ncell */
  const double *V;        /* ncell */
  const uint8_t *thick;   /* ncell, may be NULL */
  int nlam;
  const double *lam, *nu; /* nlam */
  const double *KabsTot;  /* ncell*nlam */
  const double *KscaTot;  /* ncell*nlam */
  const double *KpCell;   /* ncell*(TMAX+1): sum_grains Kp w wopac */
  int kp_uniform;         /* 1: KpCell has one row shared by all cells */
  const double *BB;       /* nlam*(TMAX+1) */
  const double *Fstar;    /* nlam */
  double Lstar;
  /* scattering: nmix mixtures of grain/opac components.  For each cell the
   * scattering component is chosen from ncomp components with weights
   * comp_w[c*ncomp + q] * Ksca_comp[q*nlam + l]. */
  int ncomp;
  const double *comp_w;    /* ncell*ncomp (w(ii)*wopac(ii,iopac)) */
  const double *Ksca_comp; /* ncomp*nlam */
  const double *F_comp;    /* ncomp*nlam*6*180 (F11,F12,F22,F33,F34,F44) */
  const double *IF_comp;   /* ncomp*nlam*2 (IF11, IF12) */
  const double *sinthet;   /* 180: sin(pi*(i-0.5)/180) */
  const double *cos2phi;   /* 361 */
  const double *sin2phi;   /* 361 */
  /* random walk: per-cell diffusion tables, or NULL to evaluate
   * DiffCoeffCell lazily per cell as the reference does (g_comp needed) */
  const double *KDext;     /* ncell*(TMAX+1) or NULL */
  const double *KDabs;     /* ncell*(TMAX+1) or NULL */
  const double *g_comp;    /* ncomp*nlam asymmetry parameters, for lazy tables */
  const double *rw_y;      /* 1000 */
  const double *rw_phi;    /* 1000 */
} orc_model;

typedef struct {
  int64_t nphot;
  uint64_t seed;
  int scat_how;     /* 0 none, 1 isotropic, 2 full Mueller */
  int randomwalk;   /* RNDW */
  double factRW;
  int64_t maxinteract; /* 0 = no overflow roulette */
  int rng;          /* 0 = Philox per packet (GPU streams), 1 = ran1 (Subroutines.f:1481) */
  int32_t idum;     /* ran1 seed when rng == 1 */
} orc_run;

typedef struct {
  double *EJv, *EJv2, *Eabs, *T; /* ncell */
  int32_t *Ni;                   /* ncell */
  double *spec;                  /* nlam*31 */
  double *scatspec;              /* nlam*31 */
  int32_t *ispec;                /* nlam*31 */
  /* counters: 0 emitted, 1 interactions, 2 absorptions, 3 scatterings,
   * 4 random-walk steps, 5 star hits (re-launched), 6 abandoned traces,
   * 7 overflow kills, 8 cell crossings, 9 escapes */
  int64_t counters[16];
  double tautot;
  int32_t *Nabs;                 /* ncell: absorption events (may be NULL) */
} orc_result;

int orc_mcradiation(const orc_model *m, const orc_run *run, orc_result *out);

/* temperature from absorbed energy per mass, Radiation.f:629-702 (used for
 * the post-MC step Main.f:498-549) */
double orc_determine_t(const double *kp, double E1, double Tcur);
/* 1: orc_determine_t and orc_increase_t (and the packet loop through them)
 * form real(i)**4 in single precision as the reference does; 0: FP64 */
void orc_set_t4_single(int on);
/* Bjorkman-Wood upward scan, Radiation.f:537-562 */
double orc_increase_t(const double *kp, double E1, double Tcur);

/* Diffuse (Diffusion.f:9-330) on the dense system with DGESV's elimination.
 * KDext: ncell*(TMAX+1) DiffCoeffCell tables (orc_diffcoeff_cell); KpCell as
 * in orc_model; thick: InitRandomWalk flags, cleared in place as
 * Diffusion.f:136 does; T in/out; EJv written for the solved cells.
 * stats: [0] cells selected, [1] unknowns, [2] cells solved in the last pass,
 * [3] passes whose DGESV returned INFO > 0. */
int orc_diffuse(int nr, int nt, const double *R, const double *Theta, const double *dens, int ncomp,
                const double *comp_w, const double *KDext, const double *KpCell, int kp_uniform, uint8_t *thick,
                int nphotmin, double dtmax, const int32_t *Ni, const double *dT, double *T, double *EJv,
                int *stats);

/* DiskStructure (DiskStructure.f:85-468) for 'DISK' grains with
 * CheckMinimumDensity and CheckCells.  zones: 7 values per zone (rin, rout
 * [AU], sh, rsh, shpow, denspow, fix_struct as 0/1); shscale (nR) and
 * grain_scale (ng*nR) may be NULL.  Cell arrays in/out as mcg_disk_structure. */
/* one scattered-light field of the ray tracer (TraceMono, TraceMono.f:583-
 * 914) at lam0 for inclination angle, nphot Monte Carlo and nstar starlight
 * packets with Philox key `key`; SF laid out as mcg_scatter_field's;
 * info: [0] nsub, [1] geometry failures, [2] interaction-cap kills, [3]
 * packets with no start.  Kabs_c, Ksca_c: ncomp*nlam; T per cell. */
int orc_scatter_field(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, int scat_how,
                      double angle, double lam0, int64_t nphot, int64_t nstar, uint64_t key, int nexits, double *SF,
                      int64_t *info);

int orc_disk_structure(int nR, int nTheta, int ng, const double *R, const double *Theta, const double *V,
                       double Mstar, int nzones, const double *zones, const double *shscale,
                       const double *grain_scale, const int *shtype, const double *Temp, double *dens,
                       double *dens0, double *gasdens, double *w, double *w0);

/* Ray-traced spectrum without a scattering field (TracePath + TraceFlux,
 * TraceMono.f:2032-2297 and 8-497): Kabs_c, Ksca_c per component (ncomp*nlam),
 * T per cell; the model's dens is used as given.  info: [0] image radii,
 * [1] rays ended by a geometry failure. */
/* the scattered-light field settings of the ray tracer (0 packets: none) */
typedef struct {
  int64_t nphot, nstar;
  uint64_t seed;
  int nexits;
} orc_scat_opts;

int orc_trace_spectrum_scat(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T,
                            int scat_how, double angle, int nphi, int nj0, int nRfix, const double *Rfix,
                            double lam_path, int tracestar, double dimstar, int nobs, const double *lam_obs,
                            double *flux, int *info, const orc_scat_opts *so);
int orc_trace_image_scat(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T,
                         int scat_how, double angle, int nphi, int nj0, int nRfix, const double *Rfix, int tracestar,
                         double dimstar, double lam0, int npix, int nint, double Rmax, double pa, uint64_t seed,
                         int linear, double *flux, double *im, int *info, const orc_scat_opts *so);

int orc_trace_spectrum(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T,
                       int scat_how, double angle, int nphi, int nj0, int nRfix, const double *Rfix,
                       double lam_path, int tracestar, double dimstar, int nobs, const double *lam_obs, double *flux,
                       int *info);

/* MakeImage without polarisation, planets or convolution: npix^2 image
 * im[(ix-1) npix + (iy-1)], flux[0] at lam0; the points' uniforms from
 * Philox (key seed, counter (0, 1, s_lo, s_hi)) */
int orc_trace_image(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, int scat_how,
                    double angle, int nphi, int nj0, int nRfix, const double *Rfix, int tracestar, double dimstar,
                    double lam0, int npix, int nint, double Rmax, double pa, uint64_t seed, int linear, double *flux,
                    double *im, int *info);

/* ran1 (Numerical Recipes minimal standard + shuffle), Subroutines.f:1481-1509 */
double orc_ran1(int32_t *idum, int32_t *iv, int32_t *iy);

#ifdef __cplusplus
}
#endif

#endif /* MCMAX_ORACLE_H */
