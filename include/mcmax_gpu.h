/*
 * mcmax_gpu.h -- C-ABI of the B200 (sm_100a) MCMax hot-path library
 * (libmcmax_gpu.so).
 *
 * Two reference entry points are replaced:
 *
 *   ComputePart  (ComputePart.f:1)   subroutine ComputePart(p,ii,input,amin,
 *                amax,apow,fmax,blend,porosity,inp_abun,iopac,normalize_abun,
 *                standard,nsubgrains) -- DHS/Mie opacities of one grain bin.
 *                Replaced by mcg_compute_part / mcg_compute_part_batch.  The
 *                caller passes the refractive indices already read from the
 *                .lnk files and regridded (readrefindCP, ComputePart.f:1102)
 *                and receives what ComputePart writes into p%Kabs/Ksca/Kext
 *                (iopac,:), p%F(iopac,:), p%rho(iopac), p%mscale/rscale.
 *
 *   MCRadiation  (MCRadiation.f:6)   subroutine MCRadiation(NphotTot,niter,
 *                dofastvisc) -- the photon-packet loop.  MCRadiation reads
 *                module globals (grid, densities, grain opacities, BB table);
 *                the library receives them once through mcg_set_model
 *                (mirroring what Init.f builds) and mcg_mcradiation runs the
 *                packet loop, returning C(i,j)%EJv/EJv2/Eabs/Ni/T and the
 *                MC spectra (MCRadiation.f:581-646).  NphotTot is in/out as
 *                in the reference.
 *
 *   mcg_finalize_t replaces the temperature step that follows the call
 *   (Main.f:498-549: EJv/V, EJv2/V^2, determineT, dEJv, dT), and
 *   mcg_diffuse the diffusion step after it (Diffuse, Diffusion.f:9).
 *
 * Layout conventions (all arrays are plain host pointers, row-major):
 *   cells      (i,j), i = 0..nr-1 (i = 0 is the star-to-Rin cell),
 *              j = 1..nt-1, flattened as c = i*(nt-1) + (j-1)
 *   components q = one (grain ii, opacity set iopac) pair of the reference;
 *              comp_w[c*ncomp + q] = C(i,j)%w(ii) * C(i,j)%wopac(ii,iopac)
 *   Mueller    F[((q*nlam + l)*6 + e)*180 + k], e = F11,F12,F22,F33,F34,F44
 *   BB         BB[l*(TMAX+1) + iT], TMAX = 10000 (Modules.f:5)
 *   spectra    spec[l*31 + iangle], iangle = 1..30 (MCRadiation.f:20)
 *
 * Errors: every call returns mcg_status; the library never aborts the
 * process (the reference stops on e.g. MCRadiation.f:1231).  mcg_last_error
 * gives the message of the last failing call on a context.  A context is
 * used from one host thread at a time.
 */
#ifndef MCMAX_GPU_H
#define MCMAX_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCG_TMAX 10000
#define MCG_NANG 180
#define MCG_NANGLE_SED 30
#define MCG_NCOUNTERS 16

typedef enum {
  MCG_OK = 0,
  MCG_ERR_ARG = 1,     /* invalid argument (sizes, null pointers, ranges) */
  MCG_ERR_CUDA = 2,    /* a CUDA call failed */
  MCG_ERR_STATE = 3,   /* call out of order (e.g. mcradiation before set_model) */
  MCG_ERR_NOMEM = 4,   /* device allocation failed */
  MCG_ERR_LIMIT = 5,   /* a size is beyond a documented maximum */
  MCG_ERR_RUN = 6      /* the run finished with packets in an error state */
} mcg_status;

typedef struct mcg_ctx mcg_ctx;

/* Create a context on CUDA device `device`. */
mcg_status mcg_create(mcg_ctx **out, int device);
/* Release all device memory of the context. */
void mcg_destroy(mcg_ctx *ctx);
/* Message of the last failing call (empty string when none). */
const char *mcg_last_error(const mcg_ctx *ctx);
/* Library version (major*10000 + minor*100 + patch). */
int mcg_version(void);

/* ----------------------------------------------------------------------
 * ComputePart (ComputePart.f:1-552), standard = 'FILE' form.
 * -------------------------------------------------------------------- */
typedef struct {
  int nlam;
  const double *lam;   /* nlam, micron */
  int nm;              /* materials in the particle file */
  const double *e1;    /* nm*nlam: real refractive index n on the grid */
  const double *e2;    /* nm*nlam: imaginary index k (>= 0) on the grid */
  const double *frac;  /* nm: abundances as read (inp_abun already applied) */
  const double *rho;   /* nm: material densities g/cm^3 */
  double amin, amax;   /* micron */
  double apow;         /* size distribution n(a) ~ a^-apow */
  double fmax;         /* DHS maximum vacuum-core volume fraction */
  double porosity;     /* vacuum volume fraction mixed in when blend != 0 */
  double normalize_abun; /* <= 0: none (ComputePart.f:139-156) */
  int blend;           /* Bruggeman-blend materials and vacuum */
  int ns;              /* sizes per bin (nsubgrains / particle-file ns) */
  int nf;              /* DHS filling-fraction nodes */
} mcg_part_in;

typedef struct {
  double *kabs, *ksca, *kext; /* nlam, cm^2/g */
  double *F;                  /* nlam*6*180 */
  double rho_av, mscale, rscale;
  int64_t n_dhs;              /* coated-sphere evaluations */
  int64_t n_mie;              /* homogeneous-sphere evaluations */
  int64_t n_dhs_fail;         /* DHS evaluations that fell back to Mie (Err=1) */
} mcg_part_out;

/* One grain bin, as one ComputePart call. */
mcg_status mcg_compute_part(mcg_ctx *ctx, const mcg_part_in *in, mcg_part_out *out);
/* Several grain bins in one launch sequence (the per-bin loop of
 * Init.f:3365-3400 folded into one device pass). */
mcg_status mcg_compute_part_batch(mcg_ctx *ctx, int nparts, const mcg_part_in *in,
                                  mcg_part_out *out);

/* Size of the device array behind mcg_compute_part_static (64 MiB). */
#define MCG_STATIC_ARENA_BYTES (64u * 1024u * 1024u)

/* One grain bin, as mcg_compute_part, without allocating device memory.
 * No counterpart in the reference (ComputePart itself allocates nothing on a
 * GPU); it exists for host programs that must not call cudaMalloc/cudaFree:
 * a Fortran or C driver whose device memory is already handed to its own
 * pool allocator (cudaMalloc then fails or fragments the pool), and code
 * that runs while other streams do latency-critical work (cudaFree waits
 * for the whole device).  Inputs and outputs are the same host arrays as for
 * mcg_compute_part and the tables are bit-identical to it.
 *
 * All device working memory of the call lives in one static array of
 * MCG_STATIC_ARENA_BYTES that every GPU loading this library holds until the
 * process exits.  A bin is processed in chunks of wavelengths that fit the
 * array; a bin whose single wavelength needs more (many sizes times filling
 * fractions, or very large size parameters) is rejected with MCG_ERR_LIMIT
 * and a message giving the bytes it would need.  Every call looks up the
 * array's device address on the context's device (cudaGetSymbolAddress),
 * so the call stays valid after a device reset; the first lookup on a
 * device loads the library's device code, so make the first call on each
 * device before any stream capture.  Every call shares the one
 * array: calls that overlap on the same GPU (two contexts used from two
 * host threads at once) race and must be serialised by the caller; the call
 * returns only after its own work has finished. */
mcg_status mcg_compute_part_static(mcg_ctx *ctx, const mcg_part_in *in, mcg_part_out *out);

/* ----------------------------------------------------------------------
 * Model: what Init.f builds and MCRadiation reads.
 * -------------------------------------------------------------------- */
typedef struct {
  int nr;                 /* D%nR: radial cells incl. the star cell */
  int nt;                 /* D%nTheta: theta edges; cells j = 1..nt-1 */
  const double *R;        /* nr+1 radial edges in AU, R[0] = Rstar/AU */
  const double *Theta;    /* nt: cos(theta) edges, Theta[0] = 1 ... Theta[nt-1] = 0 */
  const double *SinTheta; /* nt */
  const double *dens;     /* ncell: dust density g/cm^3 */
  const double *V;        /* ncell: cell volume cm^3 */
  int ncomp;
  const double *comp_w;   /* ncell*ncomp */
} mcg_grid;

typedef struct {
  int nlam;
  const double *lam;      /* nlam, micron */
  const double *nu;       /* nlam, Hz */
  int ncomp;
  const double *Kabs;     /* ncomp*nlam, cm^2/g */
  const double *Ksca;     /* ncomp*nlam */
  const double *F;        /* ncomp*nlam*6*180 normalised Mueller elements */
  const double *BB;       /* nlam*(TMAX+1) Planck table (Init.f:2616-2622) */
  const double *Fstar;    /* nlam stellar spectrum */
  double Lstar;           /* integrate(Fstar) */
  double Tstar;           /* K, for the star-cell temperature (Main.f:545) */
  double Rstar_cm;        /* cm */
  int scat_how;           /* 0 none, 1 isotropic, 2 full Mueller (Init.f:596-611) */
} mcg_opacity;

/* Planck table BB[l*(TMAX+1)+iT] = B_nu(iT K, lam[l]) with the reference's
 * quad-precision exponential (Init.f:2616-2622, Subroutines.f:4-21); host
 * side, needs no context. */
mcg_status mcg_bb_table(int nlam, const double *lam, double *BB);
/* one Planck value, B_nu(T, lam) in erg/s/cm^2/Hz/sr, lam in micron */
double mcg_planck(double T, double lam);

/* Upload grid and opacities and build the device tables (per-cell
 * KabsTot/KscaTot, Planck means, Mueller normalisations IF11/IF12, g,
 * random-walk diffusion tables).  Replaces the previous model. */
mcg_status mcg_set_model(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac);

/* Transport forms.  EXACT keeps the reference's evaluation order (linear
 * scans, detmath.h transcendentals): with threads = 1 it reproduces the
 * serial reference loop bit for bit.  FP64 and MIXED are the GPU-ordered
 * kernels (cumulative tables + binary search, shared-memory tables); MIXED
 * runs direction, Stokes, opacity and scattering-table arithmetic in FP32
 * and keeps positions, intersection quadratics, energies, accumulators and
 * the temperature inversion in FP64. */
typedef enum { MCG_PREC_FP64 = 0, MCG_PREC_MIXED = 1, MCG_PREC_EXACT = 2 } mcg_precision;

typedef struct {
  uint64_t seed;          /* Philox key: packet p draws stream (seed, p) */
  int randomwalk;         /* RNDW keyword 'randomwalk' */
  double factRW;          /* keyword 'factrw' (Init.f:205, default 10) */
  int64_t maxinteract;    /* > 0: overflow roulette (MCRadiation.f:568-571) */
  int nruns;              /* keyword 'nruns' (MCRadiation.f:269), >= 1: the
                             independent sub-runs execute concurrently in one
                             launch, each with its own accumulators, and are
                             averaged as the reference does */
  int precision;          /* mcg_precision */
  int threads;            /* 0: persistent grid of at most one thread per
                             1333 packets of the run (at least 256), which
                             keeps the results within the Monte Carlo noise
                             of the reference's serial packet order (a
                             packet's Bjorkman-Wood re-emissions see the
                             cell temperatures of the packets in flight with
                             it); n > 0: exactly n threads, rounded up to
                             whole blocks (1 reproduces the serial packet
                             order) */
  int block;              /* threads per block: 0 = default (256), else a
                             multiple of 32 up to 256 */
  double maxruntime;      /* keyword 'maxruntime' (Init.f:1094, default -1 =
                             off), seconds.  > 0: when a packet starts after
                             more than maxruntime seconds of the run, or once
                             a tenth of the packets have started and the run
                             projects to more than 5 maxruntime, with under 90 %
                             started, the run stops, NphotTot shrinks to
                             NphotTot (maxruntime / t) (0.5 i / Nphot) (at
                             least 10; i packets started after t seconds) and
                             the run starts over with that many packets, as
                             MCRadiation.f:323-342 does; *nphot_inout returns
                             the count that ran.  Time is measured on the
                             device from the kernel's start. */
  int32_t t4_single;      /* 1: the temperature interpolations of increaseT
                             and determineT form real(i)**4 in single
                             precision as the reference does (Radiation.f:
                             551, 584, 698), here and in the next
                             mcg_finalize_t; 0 (default): exact FP64, which
                             differs by under 1e-7 relative */
} mcg_run;

typedef struct {
  /* per-cell outputs, ncell each; NULL leaves the result on the device */
  double *EJv, *EJv2, *Eabs, *T;
  int32_t *Ni;
  /* MC spectra, nlam*31; NULL skips the copy */
  double *spec, *scatspec;
  int32_t *ispec;
  /* 0 emissions (nemit), 1 interactions, 2 absorptions, 3 scatterings,
   * 4 random-walk steps, 5 star hits, 6 abandoned traces, 7 overflow
   * kills, 8 cell crossings, 9 escapes, 10 averaged-matrix scatterings,
   * 11 geometry failures; FP64/MIXED forms with the warp scheduler, counted
   * while all 32 lanes of a warp hold packets (the bulk of the run):
   * 12 scheduled warp phases, 13 lanes served by them, 14 warp crossing
   * steps, 15 lanes that crossed in them (13/12 and 15/14 are the mean
   * lanes per phase and per crossing step) */
  int64_t counters[MCG_NCOUNTERS];
  double tautot;
  float device_ms;        /* transport kernel time of the call */
  float progress_ms[5];   /* time at which 50, 90, 99, 99.9, 100 % of the
                             packets had finished (the rest is the tail of
                             the heaviest packets) */
  int32_t *Nabs;          /* ncell: absorption events (Bjorkman-Wood
                             re-emissions) per cell, summed over the nruns
                             sub-runs; NULL skips the copy.  Not a reference
                             output: the count behind the accuracy criterion
                             "cells with >= 1e3 absorption events". */
} mcg_result;

/* The packet loop (MCRadiation.f:6-887).  *nphot_inout = NphotTot. */
mcg_status mcg_mcradiation(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot_inout,
                           mcg_result *res);

/* ----------------------------------------------------------------------
 * Many models in one launch (no counterpart in the reference, which runs
 * one model per process).  Models registered with mcg_add_model keep their
 * device tables; mcg_mcradiation_batch runs the packet loops of several of
 * them in one persistent launch (packets of all models share one work
 * counter), each model with its own run parameters, accumulators and result.
 * -------------------------------------------------------------------- */
#define MCG_BATCH_MAX 1024

typedef struct {
  int block;          /* threads per block (multiple of 32, <= 256); 0: tuned or 256 */
  int blocks_per_sm;  /* resident blocks per SM in the persistent grid; 0: tuned or 2 */
  int chunk;          /* packets a thread takes per visit of the work counter; 0: tuned or 1 */
  int autotune;       /* 1: time candidate shapes on a short trial (1/50 of the packets)
                         before the run and keep the fastest for later calls with the
                         same models and packet counts */
  int use_graph;      /* 1: capture the launch sequence (accumulator resets, the batched
                         kernel, the per-model combination) in a CUDA graph and replay it
                         on later calls with the same models, packet counts and shape */
  float device_ms;    /* out: device time of the batched launch */
} mcg_batch_opts;

/* Build the tables of a model (as mcg_set_model) and keep them; *model_id
 * names it in mcg_mcradiation_batch.  The model used by mcg_mcradiation is
 * not affected. */
mcg_status mcg_add_model(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac, int *model_id);
/* One launch over nmodels kept models: model k runs runs[k] with
 * nphot_inout[k] packets and writes results[k] (arrays as for
 * mcg_mcradiation).  All runs use the same precision (FP64 or MIXED).
 * runs[0].threads == 1 runs every packet on one thread in model order (the
 * serial order of mcg_mcradiation with threads = 1, for replay checks: the
 * same packets, equal up to floating-point contraction differences).
 * opts may be NULL (defaults); the launch shape used is written back. */
mcg_status mcg_mcradiation_batch(mcg_ctx *ctx, int nmodels, const int *model_ids, const mcg_run *runs,
                                 int64_t *nphot_inout, mcg_result *results, mcg_batch_opts *opts);

/* Temperatures from the last run (Main.f:498-549): T, dT, dEJv per cell
 * (any may be NULL).  Uses EJv/V and EJv2/V^2 of the last mcg_mcradiation. */
mcg_status mcg_finalize_t(mcg_ctx *ctx, double *T, double *dT, double *dEJv);

/* Diffuse (Diffusion.f:9-330, called as Diffuse(NPhotDiffuse, dTDiffuse)
 * from Main.f:561-563 after the temperature step): cells with fewer than
 * nphotmin packets or a relative error dT/T above dtmax that are optically
 * thick (or saw at most one packet) take their temperature from the
 * diffusion equation for T^4 over them and their neighbours, three passes.
 * The reference's defaults are nphotmin = 25, dtmax = 1 (Init.f:140-141).
 * Thick flags are InitRandomWalk's test with factRW (RandomWalk.f:172-190);
 * the clearing of Diffusion.f:136 applies inside this call only.
 * Ni, dT: per cell, from mcg_mcradiation and mcg_finalize_t of the current
 * model; T: in/out (the temperatures of mcg_finalize_t); EJv: out, may be
 * NULL, written only for the cells given a diffusion temperature (the
 * Planck-mean emission sum w*wopac*Kp(iT) the reference stores in C%EJv).
 * ncells (may be NULL): [0] cells selected, [1] unknowns of the system,
 * [2] cells solved in the last pass, [3] passes whose elimination met a zero
 * pivot (their temperatures are kept, as after DGESV's INFO > 0). */
mcg_status mcg_diffuse(mcg_ctx *ctx, int32_t nphotmin, double dtmax, double factRW, const int32_t *Ni,
                       const double *dT, double *T, double *EJv, int32_t *ncells);

/* Vertical structure (DiskStructure, DiskStructure.f:85-468, with
 * CheckMinimumDensity and CheckCells): per ring and species (gas, then each
 * grain) the density along theta from hydrostatic equilibrium in the
 * temperatures Temp (the TempAverage of DiskStructure.f:25, >= 2.7 K), by the
 * reference's adaptive Cash-Karp integration (Subroutines.f:1933-2090),
 * renormalised to the species' mass in the ring; rings inside a zone with a
 * fixed structure keep the zone's analytic profile.  A grain whose
 * scale-height type is not 'DISK' takes that type's closed-form profile
 * along theta (DiskStructure.f:248-344; MCG_SH_* below, the keyword
 * shtypeN of Init.f:920-926); MCG_SH_KEEP, the reference's unknown type,
 * keeps the grain's current densities.  Then every cell's dust and gas
 * densities and abundances are rebuilt from the profiles.  No radiation
 * pressure, gaps or halo.  Cell arrays in the cell order above, w and w0 with ngrains values
 * per cell (C%w, C%w0), all in/out: dens (C%dens), dens0 (C%dens0, the
 * condensable total), gasdens (C%gasdens, in dust-density units). */
typedef struct {
  double rin, rout;               /* AU */
  double sh, rsh, shpow, denspow; /* Zone(iz)%sh, Rsh, shpow, denspow */
  int32_t fix_struct;             /* 1: the zone keeps its analytic structure */
} mcg_zone;

typedef struct {
  int32_t nr, nt, ngrains;        /* D%nR, D%nTheta, grains */
  const double *R;                /* nr+1 radial edges, AU */
  const double *Theta;            /* nt cos(theta) edges */
  const double *V;                /* cell volumes, nr*(nt-1) */
  double Mstar;                   /* stellar mass, g */
  int32_t nzones;
  const mcg_zone *zones;
  const double *shscale;          /* nr scale-height factors per ring, or NULL (1) */
  const double *grain_scale;      /* ngrains*nr settling factors Grain(ii)%shscale(i), or NULL */
  const int32_t *shtype;          /* ngrains scale-height types MCG_SH_*, or NULL (all MCG_SH_DISK) */
} mcg_structure;

/* scale-height types (Grain(ii)%shtype): HALO and SHELL read the grain's
 * factor grain_scale directly, LOBE, JET, CYLI, CAVITY and WEDGE the
 * column's scale (shscale times grain_scale) as degrees, AU or a slope */
#define MCG_SH_DISK 0
#define MCG_SH_ZODI 1
#define MCG_SH_HALO 2
#define MCG_SH_LOBE 3
#define MCG_SH_JET 4
#define MCG_SH_SHELL 5
#define MCG_SH_CYLI 6
#define MCG_SH_CAVITY 7
#define MCG_SH_WEDGE 8
#define MCG_SH_KEEP 9

mcg_status mcg_disk_structure(mcg_ctx *ctx, const mcg_structure *s, const double *Temp, double *dens, double *dens0,
                              double *gasdens, double *w, double *w0);

/* Ray-traced spectrum at one inclination: the 'SPECTRUM' observation of
 * Telescope.f:137-160 -- TracePath (TraceMono.f:2032) once, then TraceFlux
 * (TraceMono.f:8) per wavelength -- for the thermal emission of the dust
 * (thermal contact, cell temperatures T) and the star seen through the
 * disk, on the current model, with the scattered light of TraceMono's
 * second Monte Carlo when the options ask for it (below).  A component's
 * extinction is Kabs + Ksca as uploaded.  The image has nphi
 * angles over half the plane and radii from the tau = 0.1 radius at
 * lam_path, the fixed radii Rfix, nr points per radial cell (nr < 0: one
 * point every -nr cells), 30 over the stellar disk and the outer edge.
 * flux[k] is the reference's image%flux at lam_obs[k] (0 outside the
 * wavelength grid): multiply by 1e23 / distance^2 [cm] for Jy.  info (may
 * be NULL): [0] image radii, [1] rays ended by a geometry failure. */
typedef struct {
  double angle;       /* inclination, rad */
  int32_t nphi;       /* image angles over half the plane (Telescope default 45) */
  int32_t nr;         /* image points per radial cell (default 2) */
  int32_t nRfix;      /* fixed radii: zone and gap edges inside the grid, AU */
  const double *Rfix;
  double lam_path;    /* micron; 0.55 for a spectrum */
  int32_t tracestar;  /* 1: add the star behind the disk */
  double dimstar;     /* factor on the star (1) */
  /* scattered light (TraceMono, TraceMono.f:583-914): with nphot_scatter or
   * nphot_star > 0 every wavelength of a full-Mueller model (every grid
   * wavelength around it, for isotropic scattering) gets a field from
   * nphot_star packets of single-scattered starlight (MakeStarScatter) and
   * nphot_scatter Monte Carlo packets of star and thermal light, and the
   * rays add twice its scattered source; an observation's defaults are
   * 1000 and 1000 (Telescope.f:606-607).  Both 0: no scattered light. */
  int64_t nphot_scatter;
  int64_t nphot_star;
  uint64_t seed_scatter; /* Philox key of the first field of the call; each later field takes the next key */
  int32_t nexits;        /* EmissionDistribution's exit rays per cell: 0 none, else >= 2 (observation default 5) */
} mcg_trace_opts;

mcg_status mcg_trace_spectrum(mcg_ctx *ctx, const mcg_trace_opts *opts, const double *T, int32_t nobs,
                              const double *lam_obs, double *flux, int32_t *info);

/* One scattered-light field (one TraceMono call at lam0 for the inclination
 * opts->angle, with opts' packet counts, key and nexits), for checking it:
 * field[((i nsub + off(j) + irg - 1) 2 + side) 91 + b] with ring i, row j's
 * sub-cell irg (off(j) = the sub-cells of the rows before j; a row of a
 * full-Mueller model has int((thet(j+1) - thet(j)) 270 / pi) sub-cells, at
 * least one, an isotropic model one), side 0 above the midplane, bin b = 0
 * the accumulated E v AU (half of it on each side for isotropic scattering)
 * and b = 1..90 the folded azimuth bins towards the observer
 * (makescattfield, TraceMono.f:1416-1497).  cap: doubles field can hold;
 * field may be NULL to ask for the size.  info: [0] nsub, [1] doubles of
 * the field, [2] packets ended by a geometry failure, [3] packets ended by
 * the interaction cap (1e6), [4] packets with no start after 1000 draws,
 * [5] the mode (0 no field, 1 isotropic, 2 angular). */
mcg_status mcg_scatter_field(mcg_ctx *ctx, const mcg_trace_opts *opts, const double *T, double lam0, double *field,
                             int64_t cap, int64_t *info);

/* Rectangular image at one wavelength: the 'IMAGE' observation of
 * Telescope.f:162-182 -- TracePath at lam0 (opts->lam_path = lam0 as the
 * reference passes it), TraceFlux at lam0, then MakeImage
 * (TraceMono.f:2759-3001) without convolution, noise, planets or
 * polarisation.  Each image cell (between two image radii and two of the
 * nphi angles) gets nint random points; at each the ray intensities are
 * interpolated (log-linear, or linear with `linear`) and
 * I * 2 pi AU^2 dR R / (nphi 2 nint) is added to the pixel of the point and
 * of its mirror below the major axis.  Pixel (ix, iy), 1-based, covers
 * x = -R cos(phi + pa), y = R sin(phi + pa) in [-Rmax, Rmax] split into
 * npixel; im[(ix-1)*npixel + (iy-1)] (the order of the reference's FITS data
 * stream) is in erg/s/Hz per pixel at unit distance: multiply by
 * 1e23 zscale / distance^2 [cm] as the reference does.  The random points
 * come from Philox4x32-10 with key `seed` and counter (0, 1, s_lo, s_hi),
 * s = (i nphi + j) nint + k the point's index (the reference draws ran2 in
 * loop order); the pixel sums are accumulated in point order.  flux[0] is
 * TraceFlux's flux at lam0.  When cap > 0, Rimg[0..nr) and rphi[nr*nphi]
 * receive the image radii (AU) and the ray intensities (radius-major);
 * cap must then be at least the number of image radii.  info (may be NULL):
 * [0] image radii, [1] rays ended by a geometry failure. */
typedef struct {
  int32_t npixel;     /* pixels per side (npix keyword, Telescope default 500) */
  int32_t nint;       /* random points per image cell (nint keyword, default 1000) */
  double Rmax;        /* half the field of view, AU */
  double pa;          /* position angle, degrees (posangle keyword) */
  uint64_t seed;      /* key of the points' random numbers */
  int32_t linear;     /* 1: linear interpolation of the intensities; 0: log-linear */
  int32_t cap;        /* capacity of Rimg in radii (0: not written) */
  double *Rimg;       /* out: image radii [cap] */
  double *rphi;       /* out: intensities [cap * nphi] */
} mcg_image_opts;

mcg_status mcg_trace_image(mcg_ctx *ctx, const mcg_trace_opts *opts, const double *T, double lam0,
                           const mcg_image_opts *io, double *flux, double *im, int32_t *info);

/* ----------------------------------------------------------------------
 * Opacity-surrogate network.  No counterpart in the reference: it stands in
 * for ComputePart's coated-sphere inner loop (ComputePart.f:318-447) inside
 * a training box (see mcg_compute_part_surrogate).  6 normalised inputs ->
 * 4 x 256 SiLU -> 64 outputs; the 256-wide layers run as BF16 tcgen05 MMAs
 * with FP32 accumulation, forward and backward.
 *
 * Parameters are one flat FP32 vector of MCG_MLP_NPARAMS values:
 *   W0[256][6], b0[256], W1..W3[3][256][256] (out, in), b1..b3[3][256],
 *   W4[64][256], b4[64].
 * -------------------------------------------------------------------- */
#define MCG_MLP_NIN 6
#define MCG_MLP_NOUT 64
#define MCG_MLP_NPARAMS 215616
#define MCG_MLP_MAX_EPOCH_LOG 256

typedef struct {
  int epochs;          /* passes over the data set */
  int batch;           /* rows per Adam step, 128 .. 2^20 */
  float lr, lr_min;    /* Adam step size, cosine decay from lr to lr_min */
  uint64_t seed;       /* shuffling */
} mcg_mlp_train_opts;

typedef struct {
  double final_loss;   /* weighted mean squared error of the last batch */
  int64_t steps;
  float device_ms;     /* training time on the device */
  double epoch_loss[MCG_MLP_MAX_EPOCH_LOG]; /* last-batch loss per epoch */
} mcg_mlp_train_report;

/* Load / read the parameters; loading also resets the optimizer state. */
mcg_status mcg_mlp_set_params(mcg_ctx *ctx, const float *params, int64_t nparams);
mcg_status mcg_mlp_get_params(mcg_ctx *ctx, float *params, int64_t nparams);
/* y[n][64] = network(x[n][6]), host arrays. */
mcg_status mcg_mlp_forward(mcg_ctx *ctx, int64_t n, const float *x, float *y);
/* Loss sum_o w[o] (y - t)^2 averaged over the n rows, and its gradient with
 * respect to every parameter (flat layout above), for one batch. */
mcg_status mcg_mlp_gradient(mcg_ctx *ctx, int64_t n, const float *x, const float *t, const float *w,
                            float *grad, double *loss);
/* Adam training on a data set of n rows (x[n][6], targets t[n][64], output
 * weights w[64]), starting from the loaded parameters. */
mcg_status mcg_mlp_train(mcg_ctx *ctx, int64_t n, const float *x, const float *t, const float *w,
                         const mcg_mlp_train_opts *opts, mcg_mlp_train_report *report);
/* Device time of one forward pass over n device-resident rows and of one
 * training step (forward, backward, Adam) on `batch` rows, each averaged
 * over `iters` repetitions after two untimed ones; the loaded parameters
 * are restored afterwards (the optimizer state is reset). */
mcg_status mcg_mlp_time(mcg_ctx *ctx, int64_t n, int iters, int batch, float *fwd_ms, float *step_ms);
/* D[128][N] = A[128][256] * B[N][256]^T on the tensor cores, BF16 inputs
 * (raw 16-bit patterns), FP32 result: a self-check of the operand layout. */
mcg_status mcg_mlp_gemm_check(mcg_ctx *ctx, int N, const uint16_t *A, const uint16_t *B, float *D);

/* ----------------------------------------------------------------------
 * ComputePart through the surrogate.  No counterpart in the reference.
 *
 * Network inputs are (log10 a [micron], log10 lambda [micron], n,
 * log10 k, porosity, fmax), each mapped from its training box to [-1, 1]:
 *   log10 a in [-2, 3], log10 lambda in [-1, log10 3000], n in [1.5, 3.5],
 *   log10 k in [-3.5, log10 2], porosity in [0, 0.6], fmax in [0, 0.8].
 * Outputs (per single grain size, physical units, see mcg_surrogate_targets):
 *   [0] log10 kappa_abs, [1] log10 kappa_sca, [2..13] moments chi_1..chi_12
 *   of F11, [14..26] moments beta_0..beta_12 of F12, [27..39] gamma_0..
 *   gamma_12 of F33, [40..52] delta_0..delta_12 of F34, [53..63] unused.
 * -------------------------------------------------------------------- */

/* Training targets: one ComputePart evaluation (same kernels and loop order
 * as mcg_compute_part) per sample in6[n][6] = (a [micron], lambda [micron],
 * n, k, porosity, fmax) for a single grain size, material density rho and
 * nf DHS filling fractions; out[n][64] as above. */
mcg_status mcg_surrogate_targets(mcg_ctx *ctx, int64_t n, const double *in6, double rho, int nf, float *out);

/* ComputePart for nparts grain bins with the loaded network in place of the
 * coated-sphere sums.  A bin qualifies when it has one material, no
 * abundance normalisation, nf == nf_train and every (size, wavelength) input
 * inside the training box; the others go through mcg_compute_part_batch
 * (the DHS/Mie kernels).  used[p] (may be NULL) = 1 when the network served
 * bin p.  Opacities are mass-weighted over the bin's sizes and scaled by
 * rho_train / rho (kappa ~ 1 / material density).  The Mueller matrix is
 * rebuilt on the 180 bins from the scattering-weighted moments in the
 * delta-M form (Wiscombe 1977): a forward fraction f = chi_12^2 / chi_11
 * (at most chi_12 and 0.99) goes into the first bin of F11 and F33, and the
 * rest comes from the series of (chi_l - f) / (1 - f), which keeps the
 * asymmetry parameter of forward-peaked grains.  F22 = F11 and F44 = F33 as
 * for spheres; F33 and F34 are scaled back where a prediction breaks
 * F12^2 + F33^2 + F34^2 <= F11^2.  F11 is normalised as ComputePart
 * normalises it (ComputePart.f:407-415). */
mcg_status mcg_compute_part_surrogate(mcg_ctx *ctx, int nparts, const mcg_part_in *in, mcg_part_out *out,
                                      double rho_train, int nf_train, int *used);

#ifdef __cplusplus
}
#endif

#endif /* MCMAX_GPU_H */
