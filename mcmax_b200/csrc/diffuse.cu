/*
 * diffuse.cu -- mcg_diffuse (Diffuse, Diffusion.f:9-330) on the device.
 *
 * The selection of cells, the stencil rows and the temperature update are
 * host logic shared with the test replay (diffuse_core.cuh).  The work that
 * grows with the model runs here:
 *   df_kd_kernel     DiffCoeffCell (Dtable.f:97-182) for a list of (cell, iT),
 *                    one thread per pair: O(nlam * ncomp) each
 *   df_fill_kernel   the stencil rows scattered into the zeroed band
 *   df_solve_kernel  banded elimination without pivoting and back
 *                    substitution, one CTA: nb steps, each a parallel
 *                    (m) x (m+1) update, m <= w (the reference's DGESV on the
 *                    dense N x N matrix is O(N^3); the band is O(nb w^2))
 *   df_kp_kernel     Planck-mean gather KpCell(c, iT)
 * The band and every device buffer of the call live for one call.
 */
#include <cuda_runtime.h>

#include <vector>

#include "diffuse_core.cuh"
#include "mcg_internal.h"

namespace {

constexpr int DF_SOLVE_THREADS = 1024;
constexpr int DF_MAX_W = 4096; /* multipliers of one step in shared memory */

__global__ void df_kd_kernel(int n, const int *cells, const int *iTs, int nlam, int ncomp, int scattering,
                             const double *comp_w, const double *g_c, const double *Ksca_c, const double *KabsTot,
                             const double *KscaTot, const double *dnu_half, const double *BB, double *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[k] = df_kd_ext(cells[k], iTs[k], nlam, ncomp, scattering, comp_w, g_c, Ksca_c, KabsTot, KscaTot, dnu_half,
                     BB);
}

__global__ void df_kp_kernel(int n, const int *cells, const int *iTs, const double *KpCell, int uniform,
                             double *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[k] = KpCell[(uniform ? (size_t)0 : (size_t)cells[k] * DF_TT) + iTs[k]];
}

__global__ void df_fill_kernel(int nb, int w, const double *coef, double *band) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nb) return;
  df_fill_row(band, w, r, coef + (size_t)r * DF_NSLOT);
}

/* One CTA.  Every thread runs the same step sequence; __syncthreads
 * separates the multipliers of a step from its update and the update from
 * the next step.  status[0] = 1 + the first step whose pivot is zero or not
 * finite (0: none). */
__global__ void __launch_bounds__(DF_SOLVE_THREADS) df_solve_kernel(int nb, int w, double *band, double *b,
                                                                     double *x, int *status) {
  extern __shared__ double lm[];
  const size_t W = 2 * (size_t)w + 1;
  for (int k = 0; k < nb; ++k) {
    if (threadIdx.x == 0 && status[0] == 0) {
      const double piv = band[(size_t)k * W + w];
      if (!(fabs(piv) > 0.0) || isinf(piv)) status[0] = k + 1;
    }
    const int m = min(w, nb - 1 - k);
    if (m <= 0) break;
    for (int t = threadIdx.x; t < m; t += blockDim.x) lm[t] = df_elim_mult(band, w, k, t);
    __syncthreads();
    const int ne = m * (m + 1);
    for (int e = threadIdx.x; e < ne; e += blockDim.x) df_elim_update(band, b, w, k, m, e, lm);
    __syncthreads();
  }
  for (int k = nb - 1; k >= 0; --k) {
    const double xk = df_back_x(band, b, w, k);
    for (int r = max(0, k - w) + (int)threadIdx.x; r < k; r += blockDim.x) df_back_update(band, b, w, k, r, xk);
    if (threadIdx.x == 0) x[k] = xk;
    __syncthreads();
  }
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

/* device buffer owned by one mcg_diffuse call */
struct DfBuf {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  ~DfBuf() { cudaFree(p); }
};

/* device backend of df_diffuse: buffers grow to the largest request */
struct DeviceBackend {
  mcg_ctx *ctx = nullptr;
  cudaStream_t st = nullptr;
  DfBuf ibuf, dbuf, band, vec;
  std::string err;

  bool fail(cudaError_t e, const char *what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  }
  bool lists(int n, const int *cells, const int *iTs, int **dc, int **dt, double **dout) {
    cudaError_t e = ibuf.ensure(sizeof(int) * 2 * (size_t)n);
    if (e == cudaSuccess) e = dbuf.ensure(sizeof(double) * (size_t)n);
    if (e != cudaSuccess) return fail(e, "diffuse: allocation");
    *dc = (int *)ibuf.p;
    *dt = *dc + n;
    *dout = (double *)dbuf.p;
    e = cudaMemcpyAsync(*dc, cells, sizeof(int) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(*dt, iTs, sizeof(int) * n, cudaMemcpyHostToDevice, st);
    return e == cudaSuccess ? true : fail(e, "diffuse: upload");
  }
  bool fetch(double *out, const double *d, int n) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? true : fail(e, "diffuse: kernel");
  }
  bool kd(int n, const int *cells, const int *iTs, double *out) {
    const DevModel &m = ctx->model;
    int *dc, *dt;
    double *d;
    if (!lists(n, cells, iTs, &dc, &dt, &d)) return false;
    df_kd_kernel<<<nblk(n, 128), 128, 0, st>>>(n, dc, dt, m.nlam, m.ncomp, m.scattering, m.comp_w, m.g_c, m.Ksca_c,
                                               m.KabsTot, m.KscaTot, m.dnu_half, m.BB, d);
    return fetch(out, d, n);
  }
  bool kp(int n, const int *cells, const int *iTs, double *out) {
    const DevModel &m = ctx->model;
    int *dc, *dt;
    double *d;
    if (!lists(n, cells, iTs, &dc, &dt, &d)) return false;
    df_kp_kernel<<<nblk(n, 256), 256, 0, st>>>(n, dc, dt, m.KpCell, m.uniform_mix, d);
    return fetch(out, d, n);
  }
  bool solve(int nb, int w, const double *coef, const double *rhs, double *x, int *code) {
    const size_t W = 2 * (size_t)w + 1;
    cudaError_t e = band.ensure(sizeof(double) * (size_t)nb * W);
    if (e == cudaSuccess) e = vec.ensure(sizeof(double) * (size_t)nb * (DF_NSLOT + 2) + sizeof(int));
    if (e != cudaSuccess) return fail(e, "diffuse: allocation of the band");
    double *dcoef = (double *)vec.p, *db = dcoef + (size_t)nb * DF_NSLOT, *dx = db + nb;
    int *dst = (int *)(dx + nb);
    e = cudaMemsetAsync(band.p, 0, sizeof(double) * (size_t)nb * W, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dst, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dcoef, coef, sizeof(double) * (size_t)nb * DF_NSLOT,
                                              cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, rhs, sizeof(double) * nb, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(e, "diffuse: upload of the rows");
    df_fill_kernel<<<nblk(nb, 256), 256, 0, st>>>(nb, w, dcoef, (double *)band.p);
    df_solve_kernel<<<1, DF_SOLVE_THREADS, sizeof(double) * (size_t)w, st>>>(nb, w, (double *)band.p, db, dx, dst);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(code, dst, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return fail(e, "diffuse: solve");
    return fetch(x, dx, nb);
  }
};

}  // namespace

mcg_status mcg_diffuse_impl(mcg_ctx *ctx, int32_t nphotmin, double dtmax, double factRW, const int32_t *Ni,
                            const double *dT, double *T, double *EJv, int32_t *ncells) {
  DevModel &m = ctx->model;
  if (!m.valid) return mcg_fail(ctx, MCG_ERR_STATE, "diffuse: no model set");
  if (!Ni || !dT || !T) return mcg_fail(ctx, MCG_ERR_ARG, "diffuse: Ni, dT and T are required");
  if (!(factRW > 0.0) || !(dtmax == dtmax)) return mcg_fail(ctx, MCG_ERR_ARG, "diffuse: factRW > 0 and a dtmax");
  if (m.nc > DF_MAX_W) return mcg_fail(ctx, MCG_ERR_ARG, "diffuse: %d theta cells, at most %d", m.nc, DF_MAX_W);
  for (int c = 0; c < m.ncell; ++c)
    if (!(T[c] >= 0.0) || !(T[c] < 1e6))
      return mcg_fail(ctx, MCG_ERR_ARG, "diffuse: T[%d] = %g is outside 0..1e6 K", c, T[c]);
  cudaStream_t st = ctx->stream;
  const int ncell = m.ncell;
  std::vector<double> R(m.nr + 1), Theta(m.nt), dens(ncell), comp_w((size_t)ncell * m.ncomp);
  MCG_CUDA(ctx, cudaMemcpyAsync(R.data(), m.R, sizeof(double) * R.size(), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(Theta.data(), m.Theta, sizeof(double) * Theta.size(), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(dens.data(), m.dens, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(comp_w.data(), m.comp_w, sizeof(double) * comp_w.size(), cudaMemcpyDeviceToHost,
                                st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  DfGrid g{m.nr, m.nt, R.data(), Theta.data(), dens.data(), m.ncomp, comp_w.data()};
  DeviceBackend be;
  be.ctx = ctx;
  be.st = st;
  DfStats stats;
  const bool ok = df_diffuse(g, be, nphotmin, dtmax, factRW, Ni, dT, T, EJv, &stats);
  if (!ok) return mcg_fail(ctx, MCG_ERR_CUDA, "%s", be.err.c_str());
  if (ncells) {
    ncells[0] = stats.ncor;
    ncells[1] = stats.nunknown;
    ncells[2] = stats.nsolved;
    ncells[3] = stats.failed;
  }
  return MCG_OK;
}
