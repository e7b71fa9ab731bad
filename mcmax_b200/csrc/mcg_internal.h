/*
 * mcg_internal.h -- shared host-side definitions of libmcmax_gpu.
 */
#ifndef MCG_INTERNAL_H
#define MCG_INTERNAL_H

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mcmax_gpu.h"

#define MCG_TT (MCG_TMAX + 1)

/* device buffer owned by a context */
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

/* Tables of the current model on the device (built by mcg_set_model). */
struct DevModel {
  bool valid = false;
  int nr = 0, nt = 0, nc = 0, ncell = 0, nlam = 0, ncomp = 0, scat_how = 0;
  int scattering = 0;       /* scat_how != 0 and some Ksca > 0 */
  int uniform_mix = 0;      /* all cells have the same comp_w row */
  double Lstar = 0.0, Tstar = 0.0, Rstar_cm = 0.0;
  double R0 = 0.0;          /* R[0], the star radius in AU */
  /* geometry */
  double *R = nullptr, *Theta = nullptr, *SinTheta = nullptr;
  double *dens = nullptr;   /* floored at 1e-50 */
  double *mass = nullptr;   /* dens*V before the floor */
  double *V = nullptr;
  double *comp_w = nullptr; /* ncell*ncomp */
  /* spectra */
  double *nu = nullptr, *dnu_half = nullptr; /* |nu_i - nu_i+1| * 0.5 */
  double *BB = nullptr;     /* nlam*TT */
  double *star_cdf = nullptr; /* nlam-1 cumulative trapezoid of Fstar */
  double *wlam = nullptr;   /* nlam SED weights */
  /* per component */
  double *Kabs_c = nullptr, *Ksca_c = nullptr, *g_c = nullptr; /* ncomp*nlam */
  double *F_c = nullptr;    /* ncomp*nlam*1080 */
  double *IF_c = nullptr;   /* ncomp*nlam*2 */
  double *Kp_c = nullptr;   /* ncomp*TT */
  /* per cell */
  double *KabsTot = nullptr, *KscaTot = nullptr; /* ncell*nlam */
  float *KabsTotF = nullptr, *KextTotF = nullptr; /* ncell*nlam, mixed path */
  double *KpCell = nullptr; /* ncell*TT (uniform mix: 1*TT) */
  /* re-emission CDF for iT0 == iT1 in a uniform mixture: TT*(nlam-1) */
  double *emit_cdf = nullptr;
  /* random walk */
  double *KDext = nullptr, *KDabs = nullptr; /* nthick_alloc*TT */
  int *kd_index = nullptr;  /* ncell -> row of KDext/KDabs or -1 */
  double *rw_dmin = nullptr; /* ncell: factRW x the shortest mean free path of the
                                cell's diffusion table (1e300 when not thick) */
  unsigned char *thick = nullptr;
  double *rw_y = nullptr, *rw_phi = nullptr; /* 1000 each */
  int kd_rows = 0;
  double kd_factRW = -1.0;  /* factRW the thick flags were built for */
  /* constant tables */
  double *sinthet = nullptr; /* 180 */
  double *cos2phi = nullptr, *sin2phi = nullptr; /* 361 */
  float *sinthetF = nullptr, *cos2phiF = nullptr, *sin2phiF = nullptr;
  /* tables of the GPU-ordered kernels (built on first use), per precision
   * index 0 = fp64, 1 = mixed */
  struct Fast {
    bool built = false;
    void *KabsRow = nullptr, *KextRow = nullptr, *Ksca_c = nullptr; /* R */
    void *KabsTotR = nullptr, *KextTotR = nullptr;                 /* R, non-uniform */
    void *scatA = nullptr, *scatB = nullptr, *F6 = nullptr;       /* R */
    unsigned char *scatG = nullptr;
  } fast[2];
  double *Ccum = nullptr;   /* uniform: TT*(nlam-1) cumulative of BB(iT)*K */
  unsigned short *emitG = nullptr; /* uniform: TMAX*32 guide table of emit_cdf rows */
  double *c2cum = nullptr, *s2cum = nullptr, *rw_logy = nullptr;
  double *KextTot = nullptr;  /* ncell*nlam, fp64 fast path, non-uniform */
  double *BBT = nullptr;      /* TT*nlam: BB temperature-major, non-uniform mixtures */
  /* host copies of the wavelength grid and the stellar spectrum */
  std::vector<double> lam_h, Fstar_h;
  std::vector<void *> owned;
};

/* Accumulators of a run on the device. */
struct DevRun {
  int ncell = 0, nlam = 0, nruns = 0;
  int t4single = 0;         /* the last run's temperature-interpolation precision, for mcg_finalize_t */
  /* per-run blocks (nruns*ncell) below; the combined results of the last
   * call are EJvTot/EJv2Tot (run averages), NiTot (sum), and the last run's
   * Eabs/T block */
  int *NiTot = nullptr;
  unsigned long long *done = nullptr, *tmark = nullptr;
  float progress_ms[5] = {0, 0, 0, 0, 0};
  double *EJv = nullptr, *EJv2 = nullptr, *Eabs = nullptr, *T = nullptr;
  int *Ni = nullptr, *lastphot = nullptr;
  double *spec = nullptr, *scatspec = nullptr;
  int *ispec = nullptr;
  unsigned long long *counters = nullptr; /* MCG_NCOUNTERS */
  double *tautot = nullptr;
  unsigned long long *next_packet = nullptr;
  /* nruns accumulation */
  double *EJvTot = nullptr, *EJv2Tot = nullptr;
  int *kp_hint = nullptr;
  /* absorption events per cell (nruns*ncell) and their sum over runs */
  int *Nabs = nullptr, *NabsTot = nullptr;
  unsigned long long *stop = nullptr; /* maxruntime record, 2 entries */
  std::vector<void *> owned;
};

struct MlpState;

struct mcg_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  DevModel model;
  DevRun run;
  bool have_run = false;
  /* reusable scratch for ComputePart */
  DevBuf part_scratch;
  /* opacity-surrogate network (created on first use) */
  MlpState *mlp = nullptr;
  /* models kept for batched runs (mcg_add_model) and their accumulators */
  std::vector<DevModel> models;
  std::vector<DevRun> runs;
  /* batched launch: device copies of the per-model kernel arguments, the
   * captured graph and the tuned launch shape */
  DevBuf batch_args;
  cudaGraphExec_t batch_graph = nullptr;
  std::vector<long long> batch_graph_key;
  int tuned_block = 0, tuned_bps = 0, tuned_chunk = 0;
  std::vector<long long> tuned_key;
};

/* kernel arguments of one prepared run: the model tables and accumulators
 * as the transport kernels see them (transport_core.cuh) */
#include "transport_core.cuh"
/* Packets in flight of a run launched with threads = 0: at most one thread
 * per MCG_PACKETS_PER_THREAD packets (and at least MCG_MIN_THREADS).  The
 * Bjorkman-Wood re-emission of a packet uses the cell temperatures of the
 * moment; in the reference's serial order a packet's whole life happens
 * between two others, while in parallel a packet trapped in an optically
 * thick cell sees the cell heated by the packets that run meanwhile.  The
 * results depart from the serial order in proportion to the share of the
 * run that is in flight at once; at one packet in flight per 1333 the
 * per-cell temperatures agree with the serial CPU run within its Monte Carlo
 * noise.  Large runs (1e8 packets) fill the GPU anyway. */
#define MCG_PACKETS_PER_THREAD 1333
#define MCG_MIN_THREADS 256
inline long long mcg_default_threads(long long nphot) {
  long long t = nphot / MCG_PACKETS_PER_THREAD;
  return t < MCG_MIN_THREADS ? MCG_MIN_THREADS : t;
}

struct RunPrep {
  TModel tm;
  TAcc ta;
  int nruns = 1;
  size_t nc = 0, ns = 0;
};

/* error helpers */
mcg_status mcg_fail(mcg_ctx *ctx, mcg_status st, const char *fmt, ...);
#define MCG_CUDA(ctx, call)                                                                     \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return mcg_fail((ctx), MCG_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                      __FILE__, __LINE__);                                                      \
  } while (0)

/* entry points implemented in the kernel translation units */
mcg_status mcg_part_batch_impl(mcg_ctx *ctx, int nparts, const mcg_part_in *in, mcg_part_out *out);
mcg_status mcg_surrogate_targets_impl(mcg_ctx *ctx, int64_t n, const double *in6, double rho, int nf, float *out);
mcg_status mcg_part_static_impl(mcg_ctx *ctx, const mcg_part_in *in, mcg_part_out *out);
mcg_status mcg_set_model_impl(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac);
mcg_status mcg_mcradiation_impl(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot, mcg_result *res);
mcg_status mcg_finalize_impl(mcg_ctx *ctx, double *T, double *dT, double *dEJv);
mcg_status mcg_trace_spectrum_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, int32_t nobs,
                                   const double *lam_obs, double *flux, int32_t *info);
mcg_status mcg_trace_image_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, double lam0,
                                const mcg_image_opts *io, double *flux, double *im, int32_t *info);
mcg_status mcg_scatter_field_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, double lam0, double *field,
                                  int64_t cap, int64_t *info);
mcg_status mcg_disk_structure_impl(mcg_ctx *ctx, const mcg_structure *s, const double *Temp, double *dens,
                                   double *dens0, double *gasdens, double *w, double *w0);
mcg_status mcg_diffuse_impl(mcg_ctx *ctx, int32_t nphotmin, double dtmax, double factRW, const int32_t *Ni,
                            const double *dT, double *T, double *EJv, int32_t *ncells);
mcg_status mcg_run_prepare(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot, RunPrep *rp, bool zero);
cudaError_t mcg_run_zero(mcg_ctx *ctx, size_t nb, size_t ns);
void mcg_run_combine(mcg_ctx *ctx, const RunPrep &rp);
mcg_status mcg_run_finish(mcg_ctx *ctx, const RunPrep &rp, float ms, mcg_result *res);
mcg_status mcg_fast_run(mcg_ctx *ctx, int precision, const void *tmodel, const void *tacc, int threads,
                        int block, float *ms);
void mcg_free_model(DevModel &m);
void mcg_free_run(DevRun &r);
void mcg_free_mlp(mcg_ctx *ctx);
mcg_status mcg_add_model_impl(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac, int *id);
mcg_status mcg_batch_impl(mcg_ctx *ctx, int n, const int *ids, const mcg_run *runs, int64_t *nphot,
                          mcg_result *res, mcg_batch_opts *opts);
void mcg_free_batch(mcg_ctx *ctx);

#endif /* MCG_INTERNAL_H */
