/*
 * transport_fast.cu -- table builders and launches of the GPU-ordered packet
 * loop (transport_fast.cuh) in its two precision forms:
 *   fp64  : R = double
 *   mixed : R = float for direction, Stokes fractions, opacities and the
 *           scattering tables; FP64 for positions, intersection quadratics,
 *           energies, accumulators and the temperature inversion.
 * Per-block shared memory holds the grid edges, the star CDF, the cumulative
 * cos/sin(2 phi) sums, the opacity rows of a uniform mixture and (when they
 * fit) the component scattering opacities.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mcg_internal.h"
#include "transport_event.cuh"

namespace {

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

/* cumulative of BB(iT)*K over the trapezoid intervals, iT = 0..TMAX */
__global__ void ccum_kernel(int nlam, const double *dnu_half, const double *BB, const double *K, double *C) {
  const int iT = blockIdx.x * blockDim.x + threadIdx.x;
  if (iT > TP_TMAX) return;
  double L = 0.0, s0 = BB[iT] * K[0];
  double *row = C + (size_t)iT * (nlam - 1);
  for (int i = 0; i < nlam - 1; ++i) {
    double s1 = BB[(size_t)(i + 1) * TP_TT + iT] * K[i + 1];
    L = L + dnu_half[i] * (s0 + s1);
    row[i] = L;
    s0 = s1;
  }
}

template <class R>
__global__ void scat_tables_kernel(int nmat, const double *F, const double *sinthet, R *A, R *B, R *F6) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nmat) return;
  const double *F11 = F + (size_t)k * 1080, *F12 = F11 + 180;
  double a = 0.0, b = 0.0;
  for (int j = 0; j < 180; ++j) {
    a += (TP_PI * sinthet[j]) * F11[j];
    b += (TP_PI * sinthet[j]) * F12[j];
    A[(size_t)k * 180 + j] = (R)a;
    B[(size_t)k * 180 + j] = (R)b;
  }
  for (int e = 0; e < 1080; ++e) F6[(size_t)k * 1080 + e] = (R)F[(size_t)k * 1080 + e];
}

template <class R>
__global__ void scat_guide_kernel(int nmat, const R *A, unsigned char *G) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nmat) return;
  const R *a = A + (size_t)k * 180;
  const R tot = a[179];
  int i = 0;
  for (int g = 0; g < F_NGUIDE; ++g) {
    const R v = tot * (R)g / (R)F_NGUIDE;
    while (i < 179 && !(a[i] > v)) ++i;
    G[(size_t)k * F_NGUIDE + g] = (unsigned char)i;
  }
}

__global__ void emit_guide_kernel(int n, const double *D, unsigned short *G) {
  const int iT = blockIdx.x * blockDim.x + threadIdx.x;
  if (iT >= TP_TMAX) return;
  const double *row = D + (size_t)iT * n;
  const double tot = row[n - 1];
  int i = 0;
  for (int g = 0; g < F_NGUIDE; ++g) {
    const double v = tot * (double)g / (double)F_NGUIDE;
    while (i < n - 1 && !(row[i] >= v)) ++i;
    G[(size_t)iT * F_NGUIDE + g] = (unsigned short)i;
  }
}

/* BBT[iT*nlam + l] = BB[l*TT + iT]: one Planck row per temperature */
__global__ void bbt_kernel(int nlam, const double *BB, double *BBT) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)TP_TT * nlam) return;
  const int iT = (int)(i / nlam), l = (int)(i % nlam);
  BBT[i] = BB[(size_t)l * TP_TT + iT];
}

template <class R>
__global__ void cast_kernel(long long n, const double *a, R *b) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) b[t] = (R)a[t];
}

template <class R>
__global__ void sum_cast_kernel(long long n, const double *a, const double *b, R *c) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) c[t] = (R)(a[t] + b[t]);
}

/* shared-memory layout of one block */
struct SmemPlan {
  size_t off_R, off_Th, off_ST, off_cdf, off_c2, off_s2, off_ka, off_ke, off_ks, bytes;
  bool ksca_in_smem;
};

template <class R>
SmemPlan plan_smem(int nr, int nt, int nlam, int ncomp, bool uniform) {
  SmemPlan p;
  size_t o = 0;
  p.off_R = o; o += (size_t)(nr + 1) * 8;
  p.off_Th = o; o += (size_t)nt * 8;
  p.off_ST = o; o += (size_t)nt * 8;
  p.off_cdf = o; o += (size_t)(nlam - 1) * 8;
  p.off_c2 = o; o += 181 * 8;
  p.off_s2 = o; o += 181 * 8;
  p.off_ka = o; if (uniform) o += (size_t)nlam * sizeof(R);
  o = (o + 15) & ~(size_t)15;
  p.off_ke = o; if (uniform) o += (size_t)nlam * sizeof(R);
  o = (o + 15) & ~(size_t)15;
  p.off_ks = o;
  size_t ks = (size_t)ncomp * nlam * sizeof(R);
  p.ksca_in_smem = (o + ks) <= 96 * 1024;
  if (p.ksca_in_smem) o += ks;
  p.bytes = (o + 15) & ~(size_t)15;
  return p;
}

#ifndef F_BLOCK
#define F_BLOCK 256
#endif
/* two 256-thread blocks per SM (128 registers a thread): the packet loop is
 * latency bound, and 16 resident warps per SM finish the bulk of a run 1.4x
 * sooner than 8 */
#ifndef F_MINBLOCKS
#define F_MINBLOCKS 2
#endif
/* EVENT: the warp scheduler over packet events (transport_event.cuh); the
 * block must be whole warps.  Otherwise every thread runs its packets to
 * completion one after the other (the one-thread launch replays the serial
 * packet order). */
template <class R, bool EVENT>
__global__ void __launch_bounds__(F_BLOCK, F_MINBLOCKS) transport_fast_kernel(const __grid_constant__ FModel<R> g,
                                                             const __grid_constant__ TAcc A, SmemPlan sp) {
  extern __shared__ __align__(16) unsigned char smem[];
  if (blockIdx.x == 0 && threadIdx.x == 0) A.tmark[5] = tp_globaltimer();
  double *sR = (double *)(smem + sp.off_R), *sTh = (double *)(smem + sp.off_Th), *sST = (double *)(smem + sp.off_ST);
  double *scdf = (double *)(smem + sp.off_cdf), *sc2 = (double *)(smem + sp.off_c2), *ss2 = (double *)(smem + sp.off_s2);
  R *ska = (R *)(smem + sp.off_ka), *ske = (R *)(smem + sp.off_ke), *sks = (R *)(smem + sp.off_ks);
  for (int i = threadIdx.x; i <= g.nr; i += blockDim.x) sR[i] = g.Rr[i];
  for (int i = threadIdx.x; i < g.nt; i += blockDim.x) {
    sTh[i] = g.Theta[i];
    sST[i] = g.SinTheta[i];
  }
  for (int i = threadIdx.x; i < g.nlam - 1; i += blockDim.x) scdf[i] = g.star_cdf[i];
  for (int i = threadIdx.x; i < 181; i += blockDim.x) {
    sc2[i] = g.c2cum[i];
    ss2[i] = g.s2cum[i];
  }
  if (g.uniform_mix)
    for (int i = threadIdx.x; i < g.nlam; i += blockDim.x) {
      ska[i] = g.KabsRow[i];
      ske[i] = g.KextRow[i];
    }
  if (sp.ksca_in_smem)
    for (int i = threadIdx.x; i < g.ncomp * g.nlam; i += blockDim.x) sks[i] = g.Ksca_c[i];
  __syncthreads();
  FModel<R> m = g;
  m.Rr = sR;
  m.Theta = sTh;
  m.SinTheta = sST;
  m.star_cdf = scdf;
  m.c2cum = sc2;
  m.s2cum = ss2;
  if (g.uniform_mix) {
    m.KabsRow = ska;
    m.KextRow = ske;
  }
  if (sp.ksca_in_smem) m.Ksca_c = sks;
  TLocal L;
#pragma unroll
  for (int k = 0; k < TC_N; ++k) L.cnt[k] = 0u;
  L.tautot = 0.0;
  if (EVENT) {
    fe_event_loop<R>(m, A, L);
  } else {
    const unsigned long long t0 = tp_globaltimer();
    for (;;) {
      unsigned long long pid = atomicAdd(A.next, 1ULL);
      if (pid >= (unsigned long long)m.nphot) break;
      if (tp_runtime_stop(A, m.maxruntime, m.nphot, pid, t0)) break;
      f_run_packet<R>(m, A, (int64_t)pid + m.pid0, L);
      tp_packet_done(A);
    }
  }
#pragma unroll
  for (int k = 0; k < TC_N; ++k)
    if (L.cnt[k]) atomicAdd(&A.counters[k], (unsigned long long)L.cnt[k]);
  if (L.tautot != 0.0) atomicAdd(A.tautot, L.tautot);
}

template <class R>
mcg_status build_fast_tables(mcg_ctx *ctx, int pi) {
  DevModel &m = ctx->model;
  DevModel::Fast &f = m.fast[pi];
  if (f.built) return MCG_OK;
  cudaStream_t st = ctx->stream;
  const int nlam = m.nlam, ncomp = m.ncomp, ncell = m.ncell, nmat = ncomp * nlam;
  auto alloc = [&](size_t bytes, void **p) {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) m.owned.push_back(*p);
    return e;
  };
  cudaError_t e = cudaSuccess;
  if (!m.c2cum) {
    std::vector<double> c2(181), s2(181), ly(TP_NY), y(TP_NY), cp(361), sp(361);
    MCG_CUDA(ctx, cudaMemcpy(cp.data(), m.cos2phi, 361 * 8, cudaMemcpyDeviceToHost));
    MCG_CUDA(ctx, cudaMemcpy(sp.data(), m.sin2phi, 361 * 8, cudaMemcpyDeviceToHost));
    MCG_CUDA(ctx, cudaMemcpy(y.data(), m.rw_y, TP_NY * 8, cudaMemcpyDeviceToHost));
    c2[0] = s2[0] = 0.0;
    for (int k = 1; k <= 180; ++k) {
      c2[k] = c2[k - 1] + cp[k];
      s2[k] = s2[k - 1] + sp[k];
    }
    for (int i = 0; i < TP_NY; ++i) ly[i] = std::log(y[i]);
    if ((e = alloc(181 * 8, (void **)&m.c2cum)) != cudaSuccess || (e = alloc(181 * 8, (void **)&m.s2cum)) != cudaSuccess ||
        (e = alloc(TP_NY * 8, (void **)&m.rw_logy)) != cudaSuccess)
      return mcg_fail(ctx, MCG_ERR_NOMEM, "fast tables: %s", cudaGetErrorString(e));
    MCG_CUDA(ctx, cudaMemcpyAsync(m.c2cum, c2.data(), 181 * 8, cudaMemcpyHostToDevice, st));
    MCG_CUDA(ctx, cudaMemcpyAsync(m.s2cum, s2.data(), 181 * 8, cudaMemcpyHostToDevice, st));
    MCG_CUDA(ctx, cudaMemcpyAsync(m.rw_logy, ly.data(), TP_NY * 8, cudaMemcpyHostToDevice, st));
    if (!m.uniform_mix) {
      if ((e = alloc((size_t)TP_TT * nlam * 8, (void **)&m.BBT)) != cudaSuccess)
        return mcg_fail(ctx, MCG_ERR_NOMEM, "fast tables: %s", cudaGetErrorString(e));
      bbt_kernel<<<nblk((long long)TP_TT * nlam, 256), 256, 0, st>>>(nlam, m.BB, m.BBT);
    }
    if (m.uniform_mix) {
      if ((e = alloc((size_t)TP_TT * (nlam - 1) * 8, (void **)&m.Ccum)) != cudaSuccess)
        return mcg_fail(ctx, MCG_ERR_NOMEM, "fast tables: %s", cudaGetErrorString(e));
      ccum_kernel<<<nblk(TP_TT, 256), 256, 0, st>>>(nlam, m.dnu_half, m.BB, m.KabsTot, m.Ccum);
      if ((e = alloc((size_t)TP_TMAX * F_NGUIDE * 2, (void **)&m.emitG)) != cudaSuccess)
        return mcg_fail(ctx, MCG_ERR_NOMEM, "fast tables: %s", cudaGetErrorString(e));
      emit_guide_kernel<<<nblk(TP_TMAX, 256), 256, 0, st>>>(nlam - 1, m.emit_cdf, m.emitG);
    }
  }
  const size_t rs = sizeof(R);
  if ((e = alloc((size_t)nlam * rs, &f.KabsRow)) != cudaSuccess || (e = alloc((size_t)nlam * rs, &f.KextRow)) != cudaSuccess ||
      (e = alloc((size_t)nmat * rs, &f.Ksca_c)) != cudaSuccess ||
      (e = alloc((size_t)nmat * 180 * rs, &f.scatA)) != cudaSuccess ||
      (e = alloc((size_t)nmat * 180 * rs, &f.scatB)) != cudaSuccess ||
      (e = alloc((size_t)nmat * 1080 * rs, &f.F6)) != cudaSuccess ||
      (e = alloc((size_t)nmat * F_NGUIDE, (void **)&f.scatG)) != cudaSuccess)
    return mcg_fail(ctx, MCG_ERR_NOMEM, "fast tables: %s", cudaGetErrorString(e));
  cast_kernel<R><<<nblk(nlam, 256), 256, 0, st>>>(nlam, m.KabsTot, (R *)f.KabsRow);
  sum_cast_kernel<R><<<nblk(nlam, 256), 256, 0, st>>>(nlam, m.KabsTot, m.KscaTot, (R *)f.KextRow);
  cast_kernel<R><<<nblk(nmat, 256), 256, 0, st>>>(nmat, m.Ksca_c, (R *)f.Ksca_c);
  if (m.scat_how == 2)
  {
    scat_tables_kernel<R><<<nblk(nmat, 128), 128, 0, st>>>(nmat, m.F_c, m.sinthet, (R *)f.scatA, (R *)f.scatB, (R *)f.F6);
    scat_guide_kernel<R><<<nblk(nmat, 128), 128, 0, st>>>(nmat, (const R *)f.scatA, f.scatG);
  }
  if (!m.uniform_mix) {
    const long long n = (long long)ncell * nlam;
    if ((e = alloc((size_t)n * rs, &f.KabsTotR)) != cudaSuccess || (e = alloc((size_t)n * rs, &f.KextTotR)) != cudaSuccess)
      return mcg_fail(ctx, MCG_ERR_NOMEM, "fast tables: %s", cudaGetErrorString(e));
    cast_kernel<R><<<nblk(n, 256), 256, 0, st>>>(n, m.KabsTot, (R *)f.KabsTotR);
    sum_cast_kernel<R><<<nblk(n, 256), 256, 0, st>>>(n, m.KabsTot, m.KscaTot, (R *)f.KextTotR);
  }
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  f.built = true;
  return MCG_OK;
}

/* the GPU-ordered kernels' view of the current model (global pointers) */
template <class R>
void fill_fmodel(mcg_ctx *ctx, int pi, const TModel &tm, FModel<R> &g) {
  DevModel &m = ctx->model;
  DevModel::Fast &f = m.fast[pi];
  memset(&g, 0, sizeof g);
  g.nr = tm.nr; g.nt = tm.nt; g.nc = tm.nc; g.ncell = tm.ncell; g.nlam = tm.nlam; g.ncomp = tm.ncomp;
  g.scattering = tm.scattering; g.scat_how = tm.scat_how; g.uniform_mix = tm.uniform_mix; g.rw = tm.rw;
  g.factRW = tm.factRW; g.R0 = tm.R0; g.Lstar = tm.Lstar; g.Epkt = tm.Epkt; g.nruns_d = tm.nruns_d;
  g.nphot = tm.nphot; g.maxinteract = tm.maxinteract; g.pid0 = tm.pid0; g.seed = tm.seed;
  g.Rr = tm.R; g.Theta = tm.Theta; g.SinTheta = tm.SinTheta; g.star_cdf = tm.star_cdf;
  g.KabsRow = (const R *)f.KabsRow; g.KextRow = (const R *)f.KextRow; g.Ksca_c = (const R *)f.Ksca_c;
  g.c2cum = m.c2cum; g.s2cum = m.s2cum;
  g.dens = tm.dens; g.mass = tm.mass; g.wlam = tm.wlam;
  g.KabsTotR = (const R *)f.KabsTotR; g.KextTotR = (const R *)f.KextTotR; g.KabsTot = m.KabsTot;
  g.BB = m.BB; g.BBT = m.BBT; g.dnu_half = m.dnu_half; g.KpCell = m.KpCell;
  g.Ccum = m.Ccum; g.Dcum = m.emit_cdf; g.comp_w = m.comp_w;
  g.scatA = (const R *)f.scatA; g.scatB = (const R *)f.scatB; g.F6 = (const R *)f.F6; g.IF_c = m.IF_c;
  g.scatG = f.scatG; g.emitG = m.emitG;
  g.KDext = m.KDext; g.KDabs = m.KDabs; g.rw_logy = m.rw_logy; g.rw_phi = m.rw_phi;
  g.kd_index = m.kd_index; g.thick = m.thick; g.rw_dmin = m.rw_dmin;
  g.maxruntime = tm.maxruntime;
  g.t4single = tm.t4single;
}

template <class R>
mcg_status launch_fast(mcg_ctx *ctx, int pi, const TModel &tm, const TAcc &ta, int threads, int block, float *ms) {
  mcg_status s = build_fast_tables<R>(ctx, pi);
  if (s != MCG_OK) return s;
  DevModel &m = ctx->model;
  FModel<R> g;
  fill_fmodel<R>(ctx, pi, tm, g);
  SmemPlan sp = plan_smem<R>(m.nr, m.nt, m.nlam, m.ncomp, m.uniform_mix);
  /* the per-lane loop for the one-thread serial replay; the warp scheduler
   * otherwise (MCG_PACKET_LOOP=lane selects the per-lane loop for
   * comparisons) */
  const char *env = getenv("MCG_PACKET_LOOP");
  const bool event = threads != 1 && !(env && strcmp(env, "lane") == 0);
  auto kern = event ? transport_fast_kernel<R, true> : transport_fast_kernel<R, false>;
  MCG_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp.bytes));
  const int b = block > 0 ? block : F_BLOCK;
  if (event && b % 32 != 0) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: block must be a multiple of 32");
  int grid;
  if (threads > 0) {
    grid = (threads + b - 1) / b;
  } else {
    int per_sm = 0;
    MCG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, b, sp.bytes));
    grid = ctx->sm_count * std::max(per_sm, 1);
    const long long cap = (mcg_default_threads(tm.nphot) + b - 1) / b;
    if (cap < grid) grid = (int)cap;
  }
  MCG_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
  if (threads == 1)
    kern<<<1, 1, sp.bytes, ctx->stream>>>(g, ta, sp);
  else
    kern<<<grid, b, sp.bytes, ctx->stream>>>(g, ta, sp);
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
  MCG_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  MCG_CUDA(ctx, cudaEventElapsedTime(ms, ctx->ev0, ctx->ev1));
  return MCG_OK;
}

}  // namespace

mcg_status mcg_fast_run(mcg_ctx *ctx, int precision, const void *tmodel, const void *tacc, int threads, int block,
                        float *ms) {
  const TModel &tm = *(const TModel *)tmodel;
  const TAcc &ta = *(const TAcc *)tacc;
  if (precision == 1) return launch_fast<float>(ctx, 1, tm, ta, threads, block, ms);
  return launch_fast<double>(ctx, 0, tm, ta, threads, block, ms);
}

/* ========================================================================
 * Many models in one launch (mcg_add_model, mcg_mcradiation_batch).
 *
 * Every model has its own work counter; a thread works on one model at a
 * time, taking its packets `chunk` at a time, with at most one thread per
 * MCG_PACKETS_PER_THREAD packets of the model on it (the bound of the
 * single-model launch, which keeps each model's Bjorkman-Wood temperatures
 * in the regime of the reference's serial order), and runs them with that
 * model's tables and accumulators through the same per-packet code as the
 * single-model kernel.  With one thread, packets run in model order (model
 * k owns [off[k], off[k+1]) of one counter).  A packet keeps its
 * own Philox stream (its model's seed, its number within the model), so a
 * model's packets are the same packets whether it runs alone or in a batch
 * (the two kernels are compiled separately, so FMA contraction may round a
 * few operations differently).
 * ====================================================================== */
namespace {

template <class R>
__global__ void __launch_bounds__(F_BLOCK, F_MINBLOCKS)
    transport_batch_kernel(const FModel<R> *__restrict__ models, const TAcc *__restrict__ accs,
                           const long long *__restrict__ off, int nmodels, unsigned long long *next, int chunk,
                           unsigned long long *mnext, int *mactive, const int *__restrict__ mcap) {
  __shared__ long long soff[MCG_BATCH_MAX + 1];
  for (int i = threadIdx.x; i <= nmodels; i += blockDim.x) soff[i] = off[i];
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i < nmodels; i += blockDim.x) accs[i].tmark[5] = tp_globaltimer();
  __syncthreads();
  const long long total = soff[nmodels];
  TLocal L;
  auto clear = [&]() {
#pragma unroll
    for (int k = 0; k < TC_N; ++k) L.cnt[k] = 0u;
    L.tautot = 0.0;
  };
  auto flush = [&](const TAcc &A) {
#pragma unroll
    for (int k = 0; k < TC_N; ++k)
      if (L.cnt[k]) atomicAdd(&A.counters[k], (unsigned long long)L.cnt[k]);
    if (L.tautot != 0.0) atomicAdd(A.tautot, L.tautot);
  };
  clear();
  if (gridDim.x == 1 && blockDim.x == 1) {
    /* one thread: every packet in model order (the serial order of each
     * model's single run) */
    int cur = -1;
    for (;;) {
      const unsigned long long k0 = atomicAdd(next, (unsigned long long)chunk);
      if (k0 >= (unsigned long long)total) break;
      const long long k1 = (long long)k0 + chunk < total ? (long long)k0 + chunk : total;
      for (long long k = (long long)k0; k < k1; ++k) {
        int lo = 0, hi = nmodels;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (soff[mid] <= k)
            lo = mid;
          else
            hi = mid;
        }
        if (lo != cur) {
          if (cur >= 0) flush(accs[cur]);
          clear();
          cur = lo;
        }
        const FModel<R> &m = models[lo];
        f_run_packet<R>(m, accs[lo], (int64_t)(k - soff[lo]) + m.pid0, L);
        tp_packet_done(accs[lo]);
      }
    }
    if (cur >= 0) flush(accs[cur]);
    return;
  }
  /* Every model has its own work counter and at most mcap[m] threads on it
   * at once (its packets in flight, as the single-model launch bounds them:
   * see MCG_PACKETS_PER_THREAD).  A thread joins a model with packets left
   * and room, takes its packets `chunk` at a time until none are left, and
   * moves on; it ends when no model has both. */
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int start = (int)(gt % nmodels);
  for (;;) {
    int found = -1;
    for (int t = 0; t < nmodels && found < 0; ++t) {
      const int mm = (start + t) % nmodels;
      const long long nm = soff[mm + 1] - soff[mm];
      if (*(volatile unsigned long long *)&mnext[mm] >= (unsigned long long)nm) continue;
      if (atomicAdd(&mactive[mm], 1) < mcap[mm])
        found = mm;
      else
        atomicSub(&mactive[mm], 1);
    }
    if (found < 0) break;
    const FModel<R> &m = models[found];
    const TAcc &A = accs[found];
    const long long nm = soff[found + 1] - soff[found];
    for (;;) {
      const unsigned long long k0 = atomicAdd(&mnext[found], (unsigned long long)chunk);
      if (k0 >= (unsigned long long)nm) break;
      const long long k1 = (long long)k0 + chunk < nm ? (long long)k0 + chunk : nm;
      for (long long k = (long long)k0; k < k1; ++k) {
        f_run_packet<R>(m, A, (int64_t)k + m.pid0, L);
        tp_packet_done(A);
      }
    }
    flush(A);
    clear();
    atomicSub(&mactive[found], 1);
    start = found + 1;
  }
}

/* swap kept model `id` in as the context's current model (and back) */
struct ModelSlot {
  mcg_ctx *ctx;
  int id;
  ModelSlot(mcg_ctx *c, int i) : ctx(c), id(i) {
    std::swap(ctx->model, ctx->models[id]);
    std::swap(ctx->run, ctx->runs[id]);
  }
  ~ModelSlot() {
    std::swap(ctx->model, ctx->models[id]);
    std::swap(ctx->run, ctx->runs[id]);
  }
};

struct Shape {
  int block, bps, chunk;
};

template <class R>
mcg_status batch_run_t(mcg_ctx *ctx, int pi, int n, const int *ids, const mcg_run *runs, int64_t *nphot,
                       mcg_result *res, mcg_batch_opts *opts) {
  cudaStream_t st = ctx->stream;
  /* runs[0].threads == 1: one thread takes every packet in order (the
   * serial order of the single-model kernel with threads = 1) */
  const bool serial = runs[0].threads == 1;
  const bool use_graph = opts && opts->use_graph && !serial;
  std::vector<RunPrep> rp(n);
  std::vector<FModel<R>> fm(n);
  std::vector<TAcc> ta(n);
  std::vector<long long> off(n + 1, 0);
  mcg_status s;
  for (int i = 0; i < n; ++i) {
    ModelSlot slot(ctx, ids[i]);
    if ((s = mcg_run_prepare(ctx, &runs[i], &nphot[i], &rp[i], false)) != MCG_OK) return s;
    if ((s = build_fast_tables<R>(ctx, pi)) != MCG_OK) return s;
    fill_fmodel<R>(ctx, pi, rp[i].tm, fm[i]);
    ta[i] = rp[i].ta;
    off[i + 1] = off[i] + (long long)rp[i].tm.nphot;
  }
  /* kernel arguments in one device buffer: models | accumulators | offsets | counter */
  const size_t b_fm = ((size_t)n * sizeof(FModel<R>) + 255) & ~(size_t)255;
  const size_t b_ta = ((size_t)n * sizeof(TAcc) + 255) & ~(size_t)255;
  const size_t b_off = ((size_t)(n + 1) * sizeof(long long) + 255) & ~(size_t)255;
  /* per model: work counter, threads on it, their cap */
  const size_t b_pm = (((size_t)n * (8 + 4 + 4)) + 255) & ~(size_t)255;
  const size_t need = b_fm + b_ta + b_off + 256 + b_pm;
  if (ctx->batch_args.bytes < need) {
    if (ctx->batch_graph) {
      cudaGraphExecDestroy(ctx->batch_graph);
      ctx->batch_graph = nullptr;
      ctx->batch_graph_key.clear();
    }
    if (ctx->batch_args.p) cudaFree(ctx->batch_args.p);
    ctx->batch_args.p = nullptr;
    ctx->batch_args.bytes = 0;
    cudaError_t e = cudaMalloc(&ctx->batch_args.p, need);
    if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_NOMEM, "mcradiation_batch: %s", cudaGetErrorString(e));
    ctx->batch_args.bytes = need;
  }
  unsigned char *base = (unsigned char *)ctx->batch_args.p;
  FModel<R> *d_fm = (FModel<R> *)base;
  TAcc *d_ta = (TAcc *)(base + b_fm);
  long long *d_off = (long long *)(base + b_fm + b_ta);
  unsigned long long *d_next = (unsigned long long *)(base + b_fm + b_ta + b_off);
  unsigned long long *d_mnext = (unsigned long long *)(base + b_fm + b_ta + b_off + 256);
  int *d_mactive = (int *)(d_mnext + n);
  int *d_mcap = d_mactive + n;
  {
    std::vector<int> cap(n);
    for (int i = 0; i < n; ++i) cap[i] = (int)std::min<long long>(mcg_default_threads(rp[i].tm.nphot), 1LL << 30);
    MCG_CUDA(ctx, cudaMemcpyAsync(d_mcap, cap.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  }
  MCG_CUDA(ctx, cudaMemcpyAsync(d_fm, fm.data(), (size_t)n * sizeof(FModel<R>), cudaMemcpyHostToDevice, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(d_ta, ta.data(), (size_t)n * sizeof(TAcc), cudaMemcpyHostToDevice, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(d_off, off.data(), (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));

  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  std::vector<long long> key;
  key.push_back(pi);
  for (int i = 0; i < n; ++i) {
    key.push_back(ids[i]);
    key.push_back((long long)rp[i].tm.nphot);
    key.push_back(rp[i].nruns);
  }
  /* launch shape: explicit, tuned before, tuned now, or the default */
  Shape sh{256, 2, 1};
  if (ctx->tuned_block && ctx->tuned_key == key) sh = Shape{ctx->tuned_block, ctx->tuned_bps, ctx->tuned_chunk};
  if (opts && opts->autotune && !serial && !(ctx->tuned_block && ctx->tuned_key == key)) {
    /* short trial runs: 1/50 of every model's packets (at least 200) */
    std::vector<FModel<R>> tf = fm;
    std::vector<long long> toff(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      const long long np = std::max<long long>(200, (long long)rp[i].tm.nphot / 50);
      tf[i].nphot = np;
      toff[i + 1] = toff[i] + np;
    }
    const Shape cand[] = {{256, 2, 1}, {128, 4, 1}, {256, 2, 4}, {128, 4, 4}, {256, 1, 1}};
    float best = -1.0f;
    for (const Shape &c : cand) {
      for (int i = 0; i < n; ++i) {
        ModelSlot slot(ctx, ids[i]);
        MCG_CUDA(ctx, mcg_run_zero(ctx, (size_t)rp[i].nc * rp[i].nruns, rp[i].ns));
      }
      MCG_CUDA(ctx, cudaMemcpyAsync(d_fm, tf.data(), (size_t)n * sizeof(FModel<R>), cudaMemcpyHostToDevice, st));
      MCG_CUDA(ctx, cudaMemcpyAsync(d_off, toff.data(), (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
      MCG_CUDA(ctx, cudaMemsetAsync(d_next, 0, 8, st));
      MCG_CUDA(ctx, cudaMemsetAsync(d_mnext, 0, (size_t)n * (8 + 4), st));
      MCG_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
      transport_batch_kernel<R><<<sms * c.bps, c.block, 0, st>>>(d_fm, d_ta, d_off, n, d_next, c.chunk, d_mnext,
                                                                  d_mactive, d_mcap);
      MCG_CUDA(ctx, cudaGetLastError());
      MCG_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
      MCG_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
      float ms = 0.0f;
      MCG_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
      if (best < 0.0f || ms < best) {
        best = ms;
        sh = c;
      }
    }
    ctx->tuned_block = sh.block;
    ctx->tuned_bps = sh.bps;
    ctx->tuned_chunk = sh.chunk;
    ctx->tuned_key = key;
    MCG_CUDA(ctx, cudaMemcpyAsync(d_fm, fm.data(), (size_t)n * sizeof(FModel<R>), cudaMemcpyHostToDevice, st));
    MCG_CUDA(ctx, cudaMemcpyAsync(d_off, off.data(), (size_t)(n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
  }
  if (opts && opts->block > 0) sh.block = opts->block;
  if (opts && opts->blocks_per_sm > 0) sh.bps = opts->blocks_per_sm;
  if (opts && opts->chunk > 0) sh.chunk = opts->chunk;
  if (sh.block > F_BLOCK || sh.block % 32 != 0 || sh.bps < 1 || sh.bps > 8 || sh.chunk < 1 || sh.chunk > 64)
    return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation_batch: block <= %d (multiple of 32), 1 <= blocks_per_sm <= 8, "
                    "1 <= chunk <= 64", F_BLOCK);
  key.push_back(sh.block);
  key.push_back(sh.bps);
  key.push_back(sh.chunk);

  /* the launch sequence: resets, the batched kernel, per-model combination */
  auto enqueue = [&](bool timed) -> mcg_status {
    for (int i = 0; i < n; ++i) {
      ModelSlot slot(ctx, ids[i]);
      MCG_CUDA(ctx, mcg_run_zero(ctx, (size_t)rp[i].nc * rp[i].nruns, rp[i].ns));
    }
    MCG_CUDA(ctx, cudaMemsetAsync(d_next, 0, 8, st));
    MCG_CUDA(ctx, cudaMemsetAsync(d_mnext, 0, (size_t)n * (8 + 4), st));
    if (timed) MCG_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
    if (serial)
      transport_batch_kernel<R><<<1, 1, 0, st>>>(d_fm, d_ta, d_off, n, d_next, 1, d_mnext, d_mactive, d_mcap);
    else
      transport_batch_kernel<R><<<sms * sh.bps, sh.block, 0, st>>>(d_fm, d_ta, d_off, n, d_next, sh.chunk, d_mnext,
                                                                  d_mactive, d_mcap);
    MCG_CUDA(ctx, cudaGetLastError());
    if (timed) MCG_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
    for (int i = 0; i < n; ++i) {
      ModelSlot slot(ctx, ids[i]);
      mcg_run_combine(ctx, rp[i]);
    }
    MCG_CUDA(ctx, cudaGetLastError());
    return MCG_OK;
  };
  float ms = 0.0f;
  if (use_graph) {
    if (!ctx->batch_graph || ctx->batch_graph_key != key) {
      if (ctx->batch_graph) {
        cudaGraphExecDestroy(ctx->batch_graph);
        ctx->batch_graph = nullptr;
      }
      cudaGraph_t g = nullptr;
      MCG_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      s = enqueue(false);
      cudaError_t e = cudaStreamEndCapture(st, &g);
      if (s != MCG_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
      }
      if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "mcradiation_batch: capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&ctx->batch_graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        ctx->batch_graph = nullptr;
        return mcg_fail(ctx, MCG_ERR_CUDA, "mcradiation_batch: graph: %s", cudaGetErrorString(e));
      }
      ctx->batch_graph_key = key;
    }
    MCG_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
    MCG_CUDA(ctx, cudaGraphLaunch(ctx->batch_graph, st));
    MCG_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
  } else {
    if ((s = enqueue(true)) != MCG_OK) return s;
  }
  MCG_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  MCG_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (opts) {
    opts->block = sh.block;
    opts->blocks_per_sm = sh.bps;
    opts->chunk = sh.chunk;
    opts->device_ms = ms;
  }
  mcg_status first_err = MCG_OK;
  for (int i = 0; i < n; ++i) {
    ModelSlot slot(ctx, ids[i]);
    s = mcg_run_finish(ctx, rp[i], ms, &res[i]);
    if (s != MCG_OK && first_err == MCG_OK) first_err = s;
  }
  return first_err;
}

}  // namespace

mcg_status mcg_add_model_impl(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac, int *id) {
  if (!id) return mcg_fail(ctx, MCG_ERR_ARG, "add_model: null model_id");
  if ((int)ctx->models.size() >= 65536) return mcg_fail(ctx, MCG_ERR_LIMIT, "add_model: at most 65536 kept models");
  DevModel keep_model;
  DevRun keep_run;
  const bool keep_have = ctx->have_run;
  std::swap(keep_model, ctx->model);
  std::swap(keep_run, ctx->run);
  mcg_status s = mcg_set_model_impl(ctx, grid, opac);
  if (s == MCG_OK) {
    ctx->models.push_back(DevModel());
    ctx->runs.push_back(DevRun());
    std::swap(ctx->models.back(), ctx->model);
    *id = (int)ctx->models.size() - 1;
  } else {
    mcg_free_model(ctx->model);
  }
  std::swap(keep_model, ctx->model);
  std::swap(keep_run, ctx->run);
  ctx->have_run = keep_have;
  return s;
}

mcg_status mcg_batch_impl(mcg_ctx *ctx, int n, const int *ids, const mcg_run *runs, int64_t *nphot, mcg_result *res,
                          mcg_batch_opts *opts) {
  if (n < 1 || n > MCG_BATCH_MAX || !ids || !runs || !nphot || !res)
    return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation_batch: 1 <= nmodels <= %d and non-null arrays", MCG_BATCH_MAX);
  const int prec = runs[0].precision;
  if (prec != MCG_PREC_FP64 && prec != MCG_PREC_MIXED)
    return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation_batch: precision must be FP64 or MIXED");
  for (int i = 0; i < n; ++i) {
    if (ids[i] < 0 || ids[i] >= (int)ctx->models.size())
      return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation_batch: unknown model id %d", ids[i]);
    if (runs[i].precision != prec) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation_batch: mixed precisions");
    for (int j = 0; j < i; ++j)
      if (ids[j] == ids[i]) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation_batch: model %d listed twice", ids[i]);
  }
  if (prec == MCG_PREC_MIXED) return batch_run_t<float>(ctx, 1, n, ids, runs, nphot, res, opts);
  return batch_run_t<double>(ctx, 0, n, ids, runs, nphot, res, opts);
}

void mcg_free_batch(mcg_ctx *ctx) {
  if (ctx->batch_graph) cudaGraphExecDestroy(ctx->batch_graph);
  ctx->batch_graph = nullptr;
  if (ctx->batch_args.p) cudaFree(ctx->batch_args.p);
  ctx->batch_args = DevBuf();
  for (auto &m : ctx->models) mcg_free_model(m);
  for (auto &r : ctx->runs) mcg_free_run(r);
  ctx->models.clear();
  ctx->runs.clear();
}
