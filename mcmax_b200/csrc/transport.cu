/*
 * transport.cu -- model tables, the FP64 packet-loop kernel and the
 * temperature finalisation on sm_100a.
 *
 * Table builders (what Init.f and the top of MCRadiation.f build, one thread
 * per output entry, each entry summed in the reference's order so the FP64
 * values equal the CPU oracle's):
 *   kp_comp_kernel     Kp(q,iT) = integrate(BB(:,iT) Kabs_q)      Init.f:3783-3790
 *   cell_opac_kernel   KabsTot/KscaTot(c,l) = sum_q K_q(l) w_q     MCRadiation.f:199-236
 *   kp_cell_kernel     sum_q Kp(q,iT) w_q  (computeE)              Radiation.f:611-627
 *   if_kernel          IF11/IF12 per matrix                         Init.f:3766-3776
 *   g_kernel           asymmetry parameter per matrix               Init.f:4038-4050
 *   emit_cdf_kernel    cumulative re-emission spectrum for iT0 == iT1 in a
 *                      uniform mixture (the scan of Radiation.f:966-988 done
 *                      once per temperature instead of once per absorption)
 *   kd_kernel          DiffCoeffCell per (thick cell, iT)          Dtable.f:97-182
 * Packet loop: transport_fp64_kernel (transport_core.cuh), persistent
 * threads fetching packet ids from a global counter.
 * Finalisation: finalize_kernel, Main.f:498-549.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <vector>

#include "mcg_internal.h"
#include "transport_core.cuh"

namespace {

__global__ void kp_comp_kernel(int ncomp, int nlam, const double *dnu_half, const double *BB,
                               const double *Kabs_c, double *Kp_c) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ncomp * TP_TT) return;
  const int q = (int)(t / TP_TT), iT = (int)(t % TP_TT);
  const double *K = Kabs_c + (size_t)q * nlam;
  double L = 0.0;
  double s0 = BB[iT] * K[0];
  for (int i = 0; i < nlam - 1; ++i) {
    double s1 = BB[(size_t)(i + 1) * TP_TT + iT] * K[i + 1];
    L = L + dnu_half[i] * (s0 + s1);
    s0 = s1;
  }
  Kp_c[(size_t)q * TP_TT + iT] = L;
}

__global__ void cell_opac_kernel(int ncell, int ncomp, int nlam, const double *comp_w,
                                 const double *Kabs_c, const double *Ksca_c, double *KabsTot,
                                 double *KscaTot, float *KabsF, float *KextF) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ncell * nlam) return;
  const int c = (int)(t / nlam), l = (int)(t % nlam);
  const double *w = comp_w + (size_t)c * ncomp;
  double a = 0.0, s = 0.0;
  for (int q = 0; q < ncomp; ++q) {
    a = a + Kabs_c[(size_t)q * nlam + l] * w[q];
    s = s + Ksca_c[(size_t)q * nlam + l] * w[q];
  }
  KabsTot[t] = a;
  KscaTot[t] = s;
  if (KabsF) {
    KabsF[t] = (float)a;
    KextF[t] = (float)(s + a);
  }
}

__global__ void kp_cell_kernel(int nrows, int ncomp, const double *comp_w, const double *Kp_c,
                               double *KpCell) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nrows * TP_TT) return;
  const int c = (int)(t / TP_TT), iT = (int)(t % TP_TT);
  const double *w = comp_w + (size_t)c * ncomp;
  double e = 0.0;
  for (int q = 0; q < ncomp; ++q) e = e + Kp_c[(size_t)q * TP_TT + iT] * w[q];
  KpCell[t] = e;
}

__global__ void if_kernel(int nmat, const double *F, const double *sinthet, double *IF) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nmat) return;
  const double *F11 = F + (size_t)k * 1080, *F12 = F11 + 180;
  double a = 0.0, b = 0.0;
  for (int j = 0; j < 180; ++j) {
    a = a + ((TP_PI * sinthet[j]) * F11[j]) / 180.0;
    b = b + ((TP_PI * sinthet[j]) * F12[j]) / 180.0;
  }
  IF[2 * k] = a;
  IF[2 * k + 1] = b;
}

__global__ void g_kernel(int nmat, const double *F, const double *gs, const double *gc, double *g) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nmat) return;
  const double *F11 = F + (size_t)k * 1080;
  double gg = 0.0, tot = 0.0;
  for (int ia = 0; ia < 180; ++ia) {
    gg = gg + (F11[ia] * gc[ia]) * gs[ia];
    tot = tot + F11[ia] * gs[ia];
  }
  g[k] = gg / tot;
}

__global__ void emit_cdf_kernel(int nlam, const double *dnu_half, const double *BB,
                                const double *KabsT0, double *cdf) {
  const int iT = blockIdx.x * blockDim.x + threadIdx.x;
  if (iT >= TP_TMAX) return; /* rows 0..TMAX-1 (iT0+1 <= TMAX) */
  double Lt = 0.0;
  double s0 = (BB[iT + 1] - BB[iT]) * KabsT0[0];
  double *row = cdf + (size_t)iT * (nlam - 1);
  for (int i = 0; i < nlam - 1; ++i) {
    const double *B = BB + (size_t)(i + 1) * TP_TT;
    double s1 = (B[iT + 1] - B[iT]) * KabsT0[i + 1];
    Lt = Lt + dnu_half[i] * (s0 + s1);
    row[i] = Lt;
    s0 = s1;
  }
}

/* per-cell mean asymmetry and the extinction denominator of DiffCoeffCell */
__global__ void kd_prep_kernel(int ncell, int ncomp, int nlam, int scattering, const double *comp_w,
                               const double *g_c, const double *Ksca_c, const double *KabsTot,
                               const double *KscaTot, double *den) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ncell * nlam) return;
  const int c = (int)(t / nlam), l = (int)(t % nlam);
  const double *w = comp_w + (size_t)c * ncomp;
  double g = 0.0;
  for (int q = 0; q < ncomp; ++q) g = g + (g_c[(size_t)q * nlam + l] * Ksca_c[(size_t)q * nlam + l]) * w[q];
  g = g / KscaTot[t];
  if (!scattering) g = 0.0;
  double Kext = KabsTot[t] + KscaTot[t];
  den[t] = Kext - (g * g) * KscaTot[t];
}

/* KDext/KDabs of cell rows `cells[r]` at temperatures iT = iT0 + k*diT */
__global__ void kd_kernel(int nrows, const int *cells, int nlam, const double *dnu_half,
                          const double *BB, const double *KabsTot, const double *den, int iT0,
                          int diT, int nT, double *KDext, double *KDabs, int stride) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nrows * nT) return;
  const int r = (int)(t / nT), k = (int)(t % nT);
  const int iT = iT0 + k * diT;
  const int c = cells[r];
  const double *Ka = KabsTot + (size_t)c * nlam;
  const double *D = den + (size_t)c * nlam;
  double int1 = 0.0, int2 = 0.0, int3 = 0.0;
  double b0 = BB[iT + 1] - BB[iT];
  double e0 = b0 / D[0], a0 = b0 * (Ka[0] - 0.0);
  for (int i = 0; i < nlam - 1; ++i) {
    const double *B = BB + (size_t)(i + 1) * TP_TT;
    double b1 = B[iT + 1] - B[iT];
    double e1 = b1 / D[i + 1], a1 = b1 * (Ka[i + 1] - 0.0);
    int1 = int1 + dnu_half[i] * (e0 + e1);
    int2 = int2 + dnu_half[i] * (b0 + b1);
    int3 = int3 + dnu_half[i] * (a0 + a1);
    b0 = b1;
    e0 = e1;
    a0 = a1;
  }
  KDext[(size_t)r * stride + (stride == TP_TT ? iT : k)] = int2 / int1;
  KDabs[(size_t)r * stride + (stride == TP_TT ? iT : k)] = int3 / int2;
}

__global__ void __launch_bounds__(128) transport_fp64_kernel(const __grid_constant__ TModel m,
                                                             const __grid_constant__ TAcc A) {
  if (blockIdx.x == 0 && threadIdx.x == 0) A.tmark[5] = tp_globaltimer();
  TLocal L;
#pragma unroll
  for (int k = 0; k < TC_N; ++k) L.cnt[k] = 0u;
  L.tautot = 0.0;
  const unsigned long long t0 = tp_globaltimer();
  for (;;) {
    unsigned long long pid = atomicAdd(A.next, 1ULL);
    if (pid >= (unsigned long long)m.nphot) break;
    if (tp_runtime_stop(A, m.maxruntime, m.nphot, pid, t0)) break;
    tp_run_packet(m, A, (int64_t)pid + m.pid0, L);
    tp_packet_done(A);
  }
#pragma unroll
  for (int k = 0; k < TC_N; ++k)
    if (L.cnt[k]) atomicAdd(&A.counters[k], (unsigned long long)L.cnt[k]);
  if (L.tautot != 0.0) atomicAdd(A.tautot, L.tautot);
}

}  // namespace

namespace {

__global__ void finalize_kernel(int nr, int nc, const double *V, const double *EJv, const double *EJv2,
                                const int *Ni, const double *Tbw, const double *KpCell, int uniform,
                                double Tstar_cell, int t4single, double *Tout, double *dTout,
                                double *dEJvout) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nr * nc) return;
  const int i = c / nc;
  if (i == 0) {
    Tout[c] = Tstar_cell;
    dTout[c] = 1.0;
    dEJvout[c] = 0.0;
    return;
  }
  const double *kp = KpCell + (uniform ? (size_t)0 : (size_t)c * TP_TT);
  const double e = EJv[c] / V[c];
  const double e2 = EJv2[c] / (V[c] * V[c]);
  double T = tp_determine_t(kp, e, Tbw[c], t4single);
  if (T < 1.0) T = 1.0;
  double dEJv, dT;
  if (Ni[c] > 1) {
    const double n = (double)Ni[c];
    dEJv = (e + sqrt(fabs(e2 - (e * e) / n))) / sqrt(n);
    dT = ((0.25 * T) * dEJv) / e;
  } else {
    dT = (double)TP_TMAX * 1.0;
    dEJv = kp[TP_TMAX];
  }
  if (T != T) T = 1.0;
  if (dT != dT) dT = 1.0;
  Tout[c] = T;
  dTout[c] = dT;
  dEJvout[c] = dEJv;
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

template <typename T>
T *mdev(DevModel &m, size_t n, cudaError_t &e) {
  void *p = nullptr;
  e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) m.owned.push_back(p);
  return (T *)p;
}

}  // namespace

void mcg_free_model(DevModel &m) {
  for (void *p : m.owned) cudaFree(p);
  m = DevModel();
}

void mcg_free_run(DevRun &r) {
  for (void *p : r.owned) cudaFree(p);
  r = DevRun();
}

mcg_status mcg_set_model_impl(mcg_ctx *ctx, const mcg_grid *g, const mcg_opacity *o) {
  if (!g || !o) return mcg_fail(ctx, MCG_ERR_ARG, "set_model: null grid or opacity");
  if (g->nr < 2 || g->nt < 2 || !g->R || !g->Theta || !g->SinTheta || !g->dens || !g->V || !g->comp_w)
    return mcg_fail(ctx, MCG_ERR_ARG, "set_model: nr >= 2, nt >= 2 and all grid arrays are required");
  if (o->nlam < 2 || !o->lam || !o->nu || !o->Kabs || !o->Ksca || !o->BB || !o->Fstar)
    return mcg_fail(ctx, MCG_ERR_ARG, "set_model: nlam >= 2 and all opacity arrays are required");
  if (g->ncomp < 1 || g->ncomp != o->ncomp) return mcg_fail(ctx, MCG_ERR_ARG, "set_model: ncomp mismatch");
  if (o->scat_how == 2 && !o->F) return mcg_fail(ctx, MCG_ERR_ARG, "set_model: scat_how = 2 needs F");
  if (!(o->Lstar > 0.0)) return mcg_fail(ctx, MCG_ERR_ARG, "set_model: Lstar must be > 0");
  const int nr = g->nr, nt = g->nt, nc = nt - 1, ncell = nr * nc, nlam = o->nlam, ncomp = g->ncomp;
  for (int i = 0; i < nr; ++i)
    if (!(g->R[i + 1] > g->R[i])) return mcg_fail(ctx, MCG_ERR_ARG, "set_model: radial edges must increase");
  for (int j = 0; j + 1 < nt; ++j)
    if (!(g->Theta[j + 1] < g->Theta[j])) return mcg_fail(ctx, MCG_ERR_ARG, "set_model: cos(theta) edges must decrease");
  if (g->Theta[0] != 1.0 || g->Theta[nt - 1] != 0.0)
    return mcg_fail(ctx, MCG_ERR_ARG, "set_model: Theta[0] must be 1 and Theta[nt-1] must be 0");
  for (int c = 0; c < ncell; ++c)
    if (!(g->dens[c] >= 0.0) || !(g->V[c] > 0.0))
      return mcg_fail(ctx, MCG_ERR_ARG, "set_model: densities must be >= 0 and volumes > 0 (cell %d)", c);
  for (size_t k = 0; k < (size_t)ncomp * nlam; ++k)
    if (!(o->Kabs[k] >= 0.0) || !(o->Ksca[k] >= 0.0))
      return mcg_fail(ctx, MCG_ERR_ARG, "set_model: opacities must be finite and >= 0");

  mcg_free_model(ctx->model);
  DevModel &m = ctx->model;
  m.nr = nr;
  m.nt = nt;
  m.nc = nc;
  m.ncell = ncell;
  m.nlam = nlam;
  m.ncomp = ncomp;
  m.scat_how = o->scat_how;
  m.Lstar = o->Lstar;
  m.Tstar = o->Tstar;
  m.R0 = g->R[0];
  m.Rstar_cm = o->Rstar_cm;
  m.scattering = 0;
  if (o->scat_how != 0)
    for (size_t k = 0; k < (size_t)ncomp * nlam && !m.scattering; ++k)
      for (int c = 0; c < ncell && !m.scattering; c += std::max(1, ncell / 64))
        if (o->Ksca[k] * g->comp_w[(size_t)c * ncomp + k / nlam] != 0.0) m.scattering = 1;
  m.uniform_mix = 1;
  for (int c = 1; c < ncell && m.uniform_mix; ++c)
    if (memcmp(g->comp_w, g->comp_w + (size_t)c * ncomp, sizeof(double) * ncomp) != 0) m.uniform_mix = 0;

  /* host-built small tables */
  std::vector<double> dens(ncell), mass(ncell), dnu_half(nlam - 1), star_cdf(nlam - 1), wlam(nlam);
  for (int c = 0; c < ncell; ++c) {
    mass[c] = g->dens[c] * g->V[c];
    dens[c] = g->dens[c] <= 1e-50 ? 1e-50 : g->dens[c];
  }
  for (int i = 0; i < nlam - 1; ++i) dnu_half[i] = std::fabs(o->nu[i] - o->nu[i + 1]) * 0.5;
  {
    double Lt = 0.0;
    for (int i = 0; i < nlam - 1; ++i) {
      Lt = Lt + dnu_half[i] * (o->Fstar[i] + o->Fstar[i + 1]);
      star_cdf[i] = Lt;
    }
  }
  for (int i = 0; i < nlam; ++i) {
    if (i == 0)
      wlam[i] = -1e23 / (o->nu[1] / 2.0);
    else if (i == nlam - 1)
      wlam[i] = -1e23 / ((o->nu[nlam - 1] - o->nu[nlam - 2]) / 2.0);
    else
      wlam[i] = -1e23 / ((o->nu[i + 1] - o->nu[i - 1]) / 2.0);
  }
  double sinthet[180], gs[180], gc[180], cos2phi[361], sin2phi[361];
  for (int i = 1; i <= 180; ++i) {
    sinthet[i - 1] = sin((TP_PI * ((double)i - 0.5)) / 180.0);
    gs[i - 1] = sin(TP_PI * ((double)i - 0.5) / 180.0);
    gc[i - 1] = cos(TP_PI * ((double)i - 0.5) / 180.0);
  }
  for (int i = 0; i <= 360; ++i) {
    double phi = (TP_PI * (double)(i - 1)) / 179.5;
    cos2phi[i] = cos(2.0 * phi);
    sin2phi[i] = sin(2.0 * phi);
  }
  std::vector<double> rw_y(TP_NY), rw_phi(TP_NY);
  rw_y[0] = 1.0;
  rw_phi[0] = 1.0;
  for (int i = 2; i <= TP_NY; ++i) {
    double yy = (double)(TP_NY - i + 1) / (double)(TP_NY - 1) * 0.75;
    rw_y[i - 1] = yy;
    double p = 0.0;
    for (int n = 1; n <= 1000; ++n) {
      long long e = (long long)n * n;
      double base = yy, acc = 1.0;
      while (e) {
        if (e & 1) acc *= base;
        base *= base;
        e >>= 1;
      }
      p = p + ((n + 1) % 2 == 0 ? 1.0 : -1.0) * acc;
    }
    rw_phi[i - 1] = p * 2.0;
  }

  cudaError_t e = cudaSuccess;
#define MA(T, n, name)                                                                  \
  mdev<T>(m, (size_t)(n), e);                                                           \
  if (e != cudaSuccess) {                                                               \
    mcg_free_model(m);                                                                  \
    return mcg_fail(ctx, MCG_ERR_NOMEM, "set_model: cudaMalloc(%s) failed: %s", name, cudaGetErrorString(e)); \
  }
  m.R = MA(double, nr + 1, "R");
  m.Theta = MA(double, nt, "Theta");
  m.SinTheta = MA(double, nt, "SinTheta");
  m.dens = MA(double, ncell, "dens");
  m.mass = MA(double, ncell, "mass");
  m.V = MA(double, ncell, "V");
  m.comp_w = MA(double, (size_t)ncell * ncomp, "comp_w");
  m.nu = MA(double, nlam, "nu");
  m.dnu_half = MA(double, nlam - 1, "dnu");
  m.BB = MA(double, (size_t)nlam * TP_TT, "BB");
  m.star_cdf = MA(double, nlam - 1, "star cdf");
  m.wlam = MA(double, nlam, "wlam");
  m.Kabs_c = MA(double, (size_t)ncomp * nlam, "Kabs");
  m.Ksca_c = MA(double, (size_t)ncomp * nlam, "Ksca");
  m.g_c = MA(double, (size_t)ncomp * nlam, "g");
  m.F_c = MA(double, o->F ? (size_t)ncomp * nlam * 1080 : 1, "F");
  m.IF_c = MA(double, (size_t)ncomp * nlam * 2, "IF");
  m.Kp_c = MA(double, (size_t)ncomp * TP_TT, "Kp");
  m.KabsTot = MA(double, (size_t)ncell * nlam, "KabsTot");
  m.KscaTot = MA(double, (size_t)ncell * nlam, "KscaTot");
  m.KabsTotF = MA(float, (size_t)ncell * nlam, "KabsTot f32");
  m.KextTotF = MA(float, (size_t)ncell * nlam, "KextTot f32");
  const int kprows = m.uniform_mix ? 1 : ncell;
  m.KpCell = MA(double, (size_t)kprows * TP_TT, "KpCell");
  if (m.uniform_mix) m.emit_cdf = MA(double, (size_t)TP_TMAX * (nlam - 1), "emit cdf");
  m.sinthet = MA(double, 180, "sinthet");
  m.cos2phi = MA(double, 361, "cos2phi");
  m.sin2phi = MA(double, 361, "sin2phi");
  m.rw_y = MA(double, TP_NY, "rw_y");
  m.rw_phi = MA(double, TP_NY, "rw_phi");
  m.thick = MA(unsigned char, ncell, "thick");
  m.kd_index = MA(int, ncell, "kd index");
  double *d_gs = MA(double, 180, "g sin");
  double *d_gc = MA(double, 180, "g cos");
#undef MA
  cudaStream_t st = ctx->stream;
#define UP(dst, src, n) MCG_CUDA(ctx, cudaMemcpyAsync(dst, src, (size_t)(n) * sizeof(*(dst)), cudaMemcpyHostToDevice, st))
  UP(m.R, g->R, nr + 1);
  UP(m.Theta, g->Theta, nt);
  UP(m.SinTheta, g->SinTheta, nt);
  UP(m.dens, dens.data(), ncell);
  UP(m.mass, mass.data(), ncell);
  UP(m.V, g->V, ncell);
  UP(m.comp_w, g->comp_w, (size_t)ncell * ncomp);
  UP(m.nu, o->nu, nlam);
  m.lam_h.assign(o->lam, o->lam + nlam);
  m.Fstar_h.assign(o->Fstar, o->Fstar + nlam);
  UP(m.dnu_half, dnu_half.data(), nlam - 1);
  UP(m.BB, o->BB, (size_t)nlam * TP_TT);
  UP(m.star_cdf, star_cdf.data(), nlam - 1);
  UP(m.wlam, wlam.data(), nlam);
  UP(m.Kabs_c, o->Kabs, (size_t)ncomp * nlam);
  UP(m.Ksca_c, o->Ksca, (size_t)ncomp * nlam);
  if (o->F) UP(m.F_c, o->F, (size_t)ncomp * nlam * 1080);
  UP(m.sinthet, sinthet, 180);
  UP(m.cos2phi, cos2phi, 361);
  UP(m.sin2phi, sin2phi, 361);
  UP(m.rw_y, rw_y.data(), TP_NY);
  UP(m.rw_phi, rw_phi.data(), TP_NY);
  UP(d_gs, gs, 180);
  UP(d_gc, gc, 180);
#undef UP
  MCG_CUDA(ctx, cudaMemsetAsync(m.thick, 0, ncell, st));
  MCG_CUDA(ctx, cudaMemsetAsync(m.kd_index, 0xff, sizeof(int) * ncell, st));
  const int B = 256;
  kp_comp_kernel<<<nblk((long long)ncomp * TP_TT, B), B, 0, st>>>(ncomp, nlam, m.dnu_half, m.BB, m.Kabs_c, m.Kp_c);
  cell_opac_kernel<<<nblk((long long)ncell * nlam, B), B, 0, st>>>(ncell, ncomp, nlam, m.comp_w, m.Kabs_c,
                                                                  m.Ksca_c, m.KabsTot, m.KscaTot, m.KabsTotF, m.KextTotF);
  kp_cell_kernel<<<nblk((long long)kprows * TP_TT, B), B, 0, st>>>(kprows, ncomp, m.comp_w, m.Kp_c, m.KpCell);
  if (o->F) {
    if_kernel<<<nblk((long long)ncomp * nlam, B), B, 0, st>>>(ncomp * nlam, m.F_c, m.sinthet, m.IF_c);
    g_kernel<<<nblk((long long)ncomp * nlam, B), B, 0, st>>>(ncomp * nlam, m.F_c, d_gs, d_gc, m.g_c);
  } else {
    MCG_CUDA(ctx, cudaMemsetAsync(m.IF_c, 0, sizeof(double) * ncomp * nlam * 2, st));
    MCG_CUDA(ctx, cudaMemsetAsync(m.g_c, 0, sizeof(double) * ncomp * nlam, st));
  }
  if (m.uniform_mix) emit_cdf_kernel<<<nblk(TP_TMAX, B), B, 0, st>>>(nlam, m.dnu_half, m.BB, m.KabsTot, m.emit_cdf);
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  m.valid = true;
  m.kd_factRW = -1.0;
  ctx->have_run = false;
  return MCG_OK;
}

/* largest KDext over iT of each diffusion-table row (one warp per row) */
__global__ void kd_max_kernel(int nrows, const double *KDext, double *kmax_row) {
  const int lane = threadIdx.x & 31;
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (r >= nrows) return;
  double kmax = 0.0;
  for (int iT = 1 + lane; iT <= TP_TMAX - 1; iT += 32) kmax = fmax(kmax, KDext[(size_t)r * TP_TT + iT]);
  for (int s = 16; s > 0; s >>= 1) kmax = fmax(kmax, __shfl_down_sync(0xffffffffu, kmax, s));
  if (lane == 0) kmax_row[r] = kmax;
}

/* per thick cell: factRW / (AU * max_iT KDext * dens), the bound below which
 * no random-walk jump can be taken at any temperature */
__global__ void rw_dmin_kernel(int ncell, const int *kd_index, const double *kmax_row, const double *dens,
                               double factRW, double *rw_dmin) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int r = kd_index[c];
  if (r < 0) return;
  const double kmax = kmax_row[r];
  const double lr = 1.0 / ((TP_AU * kmax) * dens[c]);
  rw_dmin[c] = kmax > 0.0 ? factRW * lr : 1e300;
}

/* thick flags (InitRandomWalk, RandomWalk.f:172-190) and the diffusion
 * tables of the thick cells for all iT.  DiffCoeffCell (Dtable.f:97-182)
 * depends on the cell only through its grain mixture (KabsTot, KscaTot and
 * the mean asymmetry), so cells with the same mixture share one row: a
 * uniform mixture needs a single row, which is what lets models with many
 * thick cells (massive disks of a parameter sweep) keep the random walk. */
static mcg_status build_rw_tables(mcg_ctx *ctx, double factRW) {
  DevModel &m = ctx->model;
  if (m.kd_factRW == factRW) return MCG_OK;
  cudaStream_t st = ctx->stream;
  const int ncell = m.ncell, nlam = m.nlam;
  cudaError_t e;
  double *den = nullptr, *kd4e = nullptr, *kd4a = nullptr;
  int *cells = nullptr;
  MCG_CUDA(ctx, cudaMalloc(&den, sizeof(double) * (size_t)ncell * nlam));
  MCG_CUDA(ctx, cudaMalloc(&kd4e, sizeof(double) * (size_t)ncell * 4));
  MCG_CUDA(ctx, cudaMalloc(&kd4a, sizeof(double) * (size_t)ncell * 4));
  MCG_CUDA(ctx, cudaMalloc(&cells, sizeof(int) * (size_t)ncell));
  std::vector<int> all(ncell);
  for (int c = 0; c < ncell; ++c) all[c] = c;
  MCG_CUDA(ctx, cudaMemcpyAsync(cells, all.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice, st));
  const int B = 256;
  kd_prep_kernel<<<nblk((long long)ncell * nlam, B), B, 0, st>>>(ncell, m.ncomp, nlam, m.scattering, m.comp_w,
                                                                m.g_c, m.Ksca_c, m.KabsTot, m.KscaTot, den);
  /* iT = 100, 600, 1100, 1600 */
  kd_kernel<<<nblk((long long)ncell * 4, B), B, 0, st>>>(ncell, cells, nlam, m.dnu_half, m.BB, m.KabsTot, den,
                                                        100, 500, 4, kd4e, kd4a, 4);
  std::vector<double> h4(ncell * 4), dens(ncell), R(m.nr + 1);
  MCG_CUDA(ctx, cudaMemcpyAsync(h4.data(), kd4e, sizeof(double) * ncell * 4, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(dens.data(), m.dens, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(R.data(), m.R, sizeof(double) * (m.nr + 1), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  const double AU = TP_AU;
  std::vector<unsigned char> thick(ncell, 0);
  std::vector<int> idx(ncell, -1), rows;
  for (int c = 0; c < ncell; ++c) {
    int i = c / m.nc;
    if (i < 1) continue;
    for (int k = 0; k < 4; ++k) {
      double lr = 1.0 / ((AU * h4[(size_t)c * 4 + k]) * dens[c]);
      if ((R[i + 1] - R[i]) > factRW * lr) thick[c] = 1;
    }
    if (thick[c]) {
      if (m.uniform_mix && !rows.empty()) {
        idx[c] = 0; /* the same mixture: the same row, bit for bit */
      } else {
        idx[c] = (int)rows.size();
        rows.push_back(c);
      }
    }
  }
  /* full tables for the thick cells */
  for (void *&p : m.owned)
    if (p == (void *)m.KDext || p == (void *)m.KDabs) {
      cudaFree(p);
      p = nullptr;
    }
  m.KDext = m.KDabs = nullptr;
  const int nrows = (int)rows.size();
  if (nrows > 0) {
    e = cudaMalloc(&m.KDext, sizeof(double) * (size_t)nrows * TP_TT);
    if (e == cudaSuccess) e = cudaMalloc(&m.KDabs, sizeof(double) * (size_t)nrows * TP_TT);
    if (e != cudaSuccess) {
      cudaFree(den); cudaFree(kd4e); cudaFree(kd4a); cudaFree(cells);
      return mcg_fail(ctx, MCG_ERR_NOMEM, "random walk: %d thick cells need %.1f GB of diffusion tables", nrows,
                      2.0 * nrows * TP_TT * 8 / 1e9);
    }
    m.owned.push_back(m.KDext);
    m.owned.push_back(m.KDabs);
    MCG_CUDA(ctx, cudaMemsetAsync(m.KDext, 0, sizeof(double) * (size_t)nrows * TP_TT, st));
    MCG_CUDA(ctx, cudaMemsetAsync(m.KDabs, 0, sizeof(double) * (size_t)nrows * TP_TT, st));
    MCG_CUDA(ctx, cudaMemcpyAsync(cells, rows.data(), sizeof(int) * nrows, cudaMemcpyHostToDevice, st));
    kd_kernel<<<nblk((long long)nrows * (TP_TMAX - 1), B), B, 0, st>>>(
        nrows, cells, nlam, m.dnu_half, m.BB, m.KabsTot, den, 1, 1, TP_TMAX - 1, m.KDext, m.KDabs, TP_TT);
  }
  MCG_CUDA(ctx, cudaMemcpyAsync(m.thick, thick.data(), ncell, cudaMemcpyHostToDevice, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(m.kd_index, idx.data(), sizeof(int) * ncell, cudaMemcpyHostToDevice, st));
  if (!m.rw_dmin) {
    e = cudaMalloc(&m.rw_dmin, sizeof(double) * (size_t)ncell);
    if (e != cudaSuccess) {
      cudaFree(den); cudaFree(kd4e); cudaFree(kd4a); cudaFree(cells);
      return mcg_fail(ctx, MCG_ERR_NOMEM, "random walk: %s", cudaGetErrorString(e));
    }
    m.owned.push_back(m.rw_dmin);
  }
  {
    std::vector<double> lim(ncell, 1e300);
    MCG_CUDA(ctx, cudaMemcpyAsync(m.rw_dmin, lim.data(), sizeof(double) * ncell, cudaMemcpyHostToDevice, st));
    MCG_CUDA(ctx, cudaStreamSynchronize(st));
  }
  if (nrows > 0) {
    /* the row maxima go into the 4-temperature buffer (no longer needed;
     * ncell*4 >= nrows entries) */
    double *kmax_row = kd4a;
    kd_max_kernel<<<nblk((long long)nrows * 32, B), B, 0, st>>>(nrows, m.KDext, kmax_row);
    rw_dmin_kernel<<<nblk(ncell, B), B, 0, st>>>(ncell, m.kd_index, kmax_row, m.dens, factRW, m.rw_dmin);
  }
  MCG_CUDA(ctx, cudaGetLastError());
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  cudaFree(den);
  cudaFree(kd4e);
  cudaFree(kd4a);
  cudaFree(cells);
  m.kd_rows = nrows;
  m.kd_factRW = factRW;
  return MCG_OK;
}

static mcg_status ensure_run_buffers(mcg_ctx *ctx, int nruns) {
  DevModel &m = ctx->model;
  DevRun &r = ctx->run;
  if (r.ncell == m.ncell && r.nlam == m.nlam && r.nruns == nruns && r.EJv) return MCG_OK;
  mcg_free_run(r);
  r.ncell = m.ncell;
  r.nlam = m.nlam;
  r.nruns = nruns;
  const size_t nc = m.ncell, nb = (size_t)m.ncell * nruns, ns = (size_t)m.nlam * (TP_NANG + 1);
  cudaError_t e = cudaSuccess;
  auto A = [&](size_t bytes) {
    void *p = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&p, std::max<size_t>(bytes, 8));
    if (e == cudaSuccess) r.owned.push_back(p);
    return p;
  };
  r.EJv = (double *)A(nb * 8);
  r.EJv2 = (double *)A(nb * 8);
  r.Eabs = (double *)A(nb * 8);
  r.T = (double *)A(nb * 8);
  r.Ni = (int *)A(nb * 4);
  r.lastphot = (int *)A(nb * 4);
  r.kp_hint = (int *)A(nb * 4);
  r.Nabs = (int *)A(nb * 4);
  r.NabsTot = (int *)A(nc * 4);
  r.stop = (unsigned long long *)A(2 * 8);
  r.EJvTot = (double *)A(nc * 8);
  r.EJv2Tot = (double *)A(nc * 8);
  r.NiTot = (int *)A(nc * 4);
  r.spec = (double *)A(ns * 8);
  r.scatspec = (double *)A(ns * 8);
  r.ispec = (int *)A(ns * 4);
  r.counters = (unsigned long long *)A(MCG_NCOUNTERS * 8);
  r.tautot = (double *)A(8);
  r.next_packet = (unsigned long long *)A(8);
  r.done = (unsigned long long *)A(8);
  r.tmark = (unsigned long long *)A(8 * 8);
  if (e != cudaSuccess) {
    mcg_free_run(r);
    return mcg_fail(ctx, MCG_ERR_NOMEM, "run buffers: %s", cudaGetErrorString(e));
  }
  return MCG_OK;
}

/* run averages in the reference's order: Tot = sum_r (EJv_r / nruns) */
__global__ static void combine_runs_kernel(int nc, int nruns, const double *EJv, const double *EJv2, const int *Ni,
                                           const int *Nabs, double *EJvTot, double *EJv2Tot, int *NiTot,
                                           int *NabsTot) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double a = 0.0, b = 0.0;
  int n = 0, na = 0;
  for (int r = 0; r < nruns; ++r) {
    a = a + EJv[(size_t)r * nc + c] / (double)nruns;
    b = b + EJv2[(size_t)r * nc + c] / (double)nruns;
    n += Ni[(size_t)r * nc + c];
    na += Nabs[(size_t)r * nc + c];
  }
  EJvTot[c] = a;
  EJv2Tot[c] = b;
  NiTot[c] = n;
  NabsTot[c] = na;
}

/* validation, run buffers and tables, zeroed accumulators and the kernel
 * arguments of one run of the current model (ctx->model / ctx->run) */
mcg_status mcg_run_prepare(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot, RunPrep *rp, bool zero) {
  if (!run || !nphot || !rp) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: null argument");
  DevModel &m = ctx->model;
  if (!m.valid) return mcg_fail(ctx, MCG_ERR_STATE, "mcradiation: mcg_set_model has not been called");
  if (*nphot < 1) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: NphotTot must be >= 1");
  const int nruns = run->nruns < 1 ? 1 : run->nruns;
  if (run->randomwalk && !(run->factRW > 0.0)) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: factRW must be > 0");
  if (run->maxinteract == 1) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: maxinteract must be 0 or > 1");
  if (run->precision != MCG_PREC_FP64 && run->precision != MCG_PREC_MIXED && run->precision != MCG_PREC_EXACT)
    return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: unknown precision %d", run->precision);
  if (run->threads < 0 || run->block < 0) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: threads/block must be >= 0");
  if (run->block > 256 || run->block % 32 != 0)
    return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: block must be 0 (default) or a multiple of 32 up to 256");
  mcg_status s;
  if ((s = ensure_run_buffers(ctx, nruns)) != MCG_OK) return s;
  if (run->randomwalk && (s = build_rw_tables(ctx, run->factRW)) != MCG_OK) return s;
  DevRun &R = ctx->run;
  const int64_t Nphot = *nphot / nruns;
  if (Nphot < 1) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: NphotTot/nruns must be >= 1");
  if (Nphot * nruns > (int64_t)2000000000)
    return mcg_fail(ctx, MCG_ERR_LIMIT, "mcradiation: at most 2e9 packets per call (packet numbers are int32)");
  const size_t nc = m.ncell, nb = (size_t)m.ncell * nruns, ns = (size_t)m.nlam * (TP_NANG + 1);
  rp->nruns = nruns;
  rp->nc = nc;
  rp->ns = ns;
  if (zero) MCG_CUDA(ctx, mcg_run_zero(ctx, nb, ns));

  TModel &tm = rp->tm;
  memset(&tm, 0, sizeof tm);
  tm.nr = m.nr; tm.nt = m.nt; tm.nc = m.nc; tm.ncell = m.ncell; tm.nlam = m.nlam; tm.ncomp = m.ncomp;
  tm.scattering = m.scattering; tm.scat_how = m.scat_how; tm.uniform_mix = m.uniform_mix;
  tm.rw = run->randomwalk ? 1 : 0;
  tm.factRW = run->factRW;
  tm.Lstar = m.Lstar;
  tm.Epkt = m.Lstar / ((double)Nphot * 1.0);
  tm.nphot = Nphot * nruns;
  tm.maxinteract = run->maxinteract;
  tm.pid0 = 0;
  tm.nruns_d = (double)nruns;
  tm.seed = run->seed;
  tm.R = m.R; tm.Theta = m.Theta; tm.SinTheta = m.SinTheta; tm.dens = m.dens; tm.mass = m.mass;
  tm.nu = m.nu; tm.dnu_half = m.dnu_half; tm.BB = m.BB; tm.star_cdf = m.star_cdf; tm.wlam = m.wlam;
  tm.KabsTot = m.KabsTot; tm.KscaTot = m.KscaTot; tm.KpCell = m.KpCell; tm.emit_cdf = m.emit_cdf;
  tm.comp_w = m.comp_w; tm.Ksca_c = m.Ksca_c; tm.F_c = m.F_c; tm.IF_c = m.IF_c;
  tm.sinthet = m.sinthet; tm.cos2phi = m.cos2phi; tm.sin2phi = m.sin2phi;
  tm.KDext = m.KDext; tm.KDabs = m.KDabs; tm.rw_y = m.rw_y; tm.rw_phi = m.rw_phi;
  tm.kd_index = m.kd_index; tm.thick = m.thick;
  tm.R0 = m.R0;
  tm.maxruntime = run->maxruntime;
  tm.t4single = run->t4_single ? 1 : 0;
  ctx->run.t4single = tm.t4single;
  TAcc &ta = rp->ta;
  memset(&ta, 0, sizeof ta);
  ta.EJv = R.EJv; ta.EJv2 = R.EJv2; ta.Eabs = R.Eabs; ta.T = R.T; ta.Ni = R.Ni; ta.lastphot = R.lastphot;
  ta.kp_hint = R.kp_hint;
  ta.spec = R.spec; ta.scatspec = R.scatspec; ta.ispec = R.ispec; ta.counters = R.counters;
  ta.tautot = R.tautot; ta.next = R.next_packet;
  ta.run_packets = Nphot;
  ta.ncell = m.ncell;
  ta.done = R.done;
  ta.tmark = R.tmark;
  ta.Nabs = R.Nabs;
  ta.stop = R.stop;
  {
    const unsigned long long tot = (unsigned long long)(Nphot * nruns);
    const double f[5] = {0.5, 0.9, 0.99, 0.999, 1.0};
    for (int k = 0; k < 5; ++k) {
      unsigned long long t = (unsigned long long)std::ceil(f[k] * (double)tot);
      ta.thresh[k] = t < 1ULL ? 1ULL : (t > tot ? tot : t);
    }
  }
  return MCG_OK;
}

/* zero the accumulators of the current run buffers (nb per-cell entries per
 * array, ns spectrum bins); capturable into a CUDA graph */
cudaError_t mcg_run_zero(mcg_ctx *ctx, size_t nb, size_t ns) {
  DevRun &R = ctx->run;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMemsetAsync(R.EJv, 0, nb * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.EJv2, 0, nb * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.Eabs, 0, nb * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.T, 0, nb * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.Ni, 0, nb * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.lastphot, 0, nb * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.kp_hint, 0, nb * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.Nabs, 0, nb * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.stop, 0, 2 * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.spec, 0, ns * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.scatspec, 0, ns * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.ispec, 0, ns * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.counters, 0, MCG_NCOUNTERS * 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.tautot, 0, 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.next_packet, 0, 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.done, 0, 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(R.tmark, 0, 8 * 8, st);
  return e;
}

/* per-run combination of the current run (nruns averages) */
void mcg_run_combine(mcg_ctx *ctx, const RunPrep &rp) {
  DevRun &R = ctx->run;
  combine_runs_kernel<<<(int)((rp.nc + 255) / 256), 256, 0, ctx->stream>>>(
      (int)rp.nc, rp.nruns, R.EJv, R.EJv2, R.Ni, R.Nabs, R.EJvTot, R.EJv2Tot, R.NiTot, R.NabsTot);
}

/* results of the current run to the caller's arrays */
mcg_status mcg_run_finish(mcg_ctx *ctx, const RunPrep &rp, float ms, mcg_result *res) {
  DevRun &R = ctx->run;
  cudaStream_t st = ctx->stream;
  const size_t nc = rp.nc, ns = rp.ns;
  MCG_CUDA(ctx, cudaGetLastError());
  res->device_ms = ms;
  unsigned long long cnt[MCG_NCOUNTERS], tmk[8];
  MCG_CUDA(ctx, cudaMemcpyAsync(cnt, R.counters, sizeof cnt, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(tmk, R.tmark, sizeof tmk, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(&res->tautot, R.tautot, 8, cudaMemcpyDeviceToHost, st));
  const size_t last = (size_t)(rp.nruns - 1) * nc;
#define DN(dst, src, n) \
  if (dst) MCG_CUDA(ctx, cudaMemcpyAsync(dst, src, (size_t)(n) * sizeof(*(dst)), cudaMemcpyDeviceToHost, st))
  DN(res->EJv, R.EJvTot, nc);
  DN(res->EJv2, R.EJv2Tot, nc);
  DN(res->Eabs, R.Eabs + last, nc);
  DN(res->T, R.T + last, nc);
  DN(res->Ni, R.NiTot, nc);
  DN(res->Nabs, R.NabsTot, nc);
  DN(res->spec, R.spec, ns);
  DN(res->scatspec, R.scatspec, ns);
  DN(res->ispec, R.ispec, ns);
#undef DN
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  for (int k = 0; k < MCG_NCOUNTERS; ++k) res->counters[k] = (int64_t)cnt[k];
  /* progress marks relative to the kernel start (tmark[5]) */
  for (int k = 0; k < 5; ++k)
    res->progress_ms[k] = (tmk[k] && tmk[5] && tmk[k] >= tmk[5]) ? (float)((double)(tmk[k] - tmk[5]) * 1e-6) : -1.0f;
  ctx->have_run = true;
  if (cnt[TC_GEOFAIL] > 0)
    return mcg_fail(ctx, MCG_ERR_RUN, "mcradiation: %llu packets found no cell boundary to hit", cnt[TC_GEOFAIL]);
  return MCG_OK;
}

static mcg_status mcg_mcradiation_once(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot, mcg_result *res,
                                       float *ms_out, bool *stopped);

mcg_status mcg_mcradiation_impl(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot, mcg_result *res) {
  if (!res) return mcg_fail(ctx, MCG_ERR_ARG, "mcradiation: null argument");
  /* maxruntime: a stopped run starts over with fewer packets (the
   * reference's `goto 6`); each restart at least halves NphotTot */
  for (int attempt = 0;; ++attempt) {
    float ms = 0.0f;
    bool stopped = false;
    mcg_status s = mcg_mcradiation_once(ctx, run, nphot, res, &ms, &stopped);
    if (s != MCG_OK || !stopped) return s;
    if (attempt >= 64) return mcg_fail(ctx, MCG_ERR_RUN, "mcradiation: maxruntime restarts did not converge");
  }
}

/* one pass of the packet loop; *stopped when maxruntime stopped it (then
 * *nphot holds the reduced count for the restart) */
static mcg_status mcg_mcradiation_once(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot, mcg_result *res,
                                       float *ms_out, bool *stopped) {
  RunPrep rp;
  mcg_status s = mcg_run_prepare(ctx, run, nphot, &rp, true);
  if (s != MCG_OK) return s;
  TModel &tm = rp.tm;
  TAcc &ta = rp.ta;
  cudaStream_t st = ctx->stream;
  const int block = run->block > 0 ? run->block : 128;
  float ms = 0.0f;
  if (run->precision == MCG_PREC_EXACT) {
    int grid;
    if (run->threads > 0) {
      grid = (run->threads + block - 1) / block;
    } else {
      int per_sm = 0;
      MCG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, transport_fp64_kernel, block, 0));
      grid = ctx->sm_count * std::max(per_sm, 1);
      const long long cap = (mcg_default_threads(tm.nphot) + block - 1) / block;
      if (cap < grid) grid = (int)cap;
    }
    MCG_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
    if (run->threads == 1)
      transport_fp64_kernel<<<1, 1, 0, st>>>(tm, ta);
    else
      transport_fp64_kernel<<<grid, block, 0, st>>>(tm, ta);
    MCG_CUDA(ctx, cudaGetLastError());
    MCG_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
    MCG_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    MCG_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  } else {
    mcg_status fs = mcg_fast_run(ctx, run->precision == MCG_PREC_MIXED ? 1 : 0, &tm, &ta, run->threads,
                                 run->block, &ms);
    if (fs != MCG_OK) return fs;
  }
  *ms_out = ms;
  if (run->maxruntime > 0.0) {
    unsigned long long rec[2] = {0ULL, 0ULL};
    MCG_CUDA(ctx, cudaMemcpyAsync(rec, ctx->run.stop, sizeof rec, cudaMemcpyDeviceToHost, st));
    MCG_CUDA(ctx, cudaStreamSynchronize(st));
    if (rec[0] != 0ULL) {
      /* NphotTot = NphotTot (maxruntime / checktime) (0.5 i / Nphot), at
       * least 10 (MCRadiation.f:333-334); i packets had started */
      const double checktime = (double)rec[1] * 1e-9 > 0.0 ? (double)rec[1] * 1e-9 : 1e-9;
      const double ntot = (double)tm.nphot;
      const double nn = (double)*nphot * (run->maxruntime / checktime) * (0.5 * (double)rec[0] / ntot);
      int64_t n = nn < 9e18 ? (int64_t)nn : *nphot;
      if (n < 10) n = 10;
      if (n >= *nphot) n = *nphot / 2 > 10 ? *nphot / 2 : 10;
      *nphot = n;
      *stopped = true;
      return MCG_OK;
    }
  }
  mcg_run_combine(ctx, rp);
  return mcg_run_finish(ctx, rp, ms, res);
}

mcg_status mcg_finalize_impl(mcg_ctx *ctx, double *T, double *dT, double *dEJv) {
  DevModel &m = ctx->model;
  DevRun &R = ctx->run;
  if (!ctx->have_run) return mcg_fail(ctx, MCG_ERR_STATE, "finalize_t: no run to finalise");
  const int nc = m.ncell;
  double *d = nullptr;
  MCG_CUDA(ctx, cudaMalloc(&d, sizeof(double) * 3 * nc));
  double R1;
  MCG_CUDA(ctx, cudaMemcpy(&R1, m.R + 1, sizeof(double), cudaMemcpyDeviceToHost));
  double x = m.Rstar_cm / (R1 * TP_AU);
  double Tsc = m.Tstar * 0.5 * (1.0 - sqrt(1.0 - x * x));
  if (Tsc < 1.0) Tsc = 1.0;
  finalize_kernel<<<nblk(nc, 256), 256, 0, ctx->stream>>>(m.nr, m.nc, m.V, R.EJvTot, R.EJv2Tot, R.NiTot,
                                                          R.T + (size_t)(R.nruns - 1) * nc, m.KpCell,
                                                          m.uniform_mix, Tsc, R.t4single, d, d + nc, d + 2 * nc);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && T) e = cudaMemcpyAsync(T, d, sizeof(double) * nc, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && dT) e = cudaMemcpyAsync(dT, d + nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && dEJv) e = cudaMemcpyAsync(dEJv, d + 2 * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "finalize_t: %s", cudaGetErrorString(e));
  return MCG_OK;
}
