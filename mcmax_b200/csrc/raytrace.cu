/*
 * raytrace.cu -- mcg_trace_spectrum: the ray-traced flux of the current
 * model at one inclination (rt_core.cuh for the algorithm and its
 * reference lines).
 *
 *   rt_cell_kernel  one thread per cell: extinction and source function at
 *                   a wavelength
 *   rt_ray_kernel   one thread per image ray (radius, angle): the path
 *                   through the cells and the formal solution
 * The image grid, the tau = 0.1 radius and the flux sum are host logic
 * shared with the test replay.
 */
#include <cuda_runtime.h>

#include <vector>

#include "mcg_internal.h"
#include "rt_core.cuh"

namespace {

constexpr int RT_MAXSTEPS = 1 << 20;

__global__ void rt_cell_kernel(int ncell, int ncomp, int nlam, const double *comp_w, const double *Kabs_c,
                               const double *Ksca_c, const double *BB, const double *T, int l1, int l2, double w1,
                               double w2, double *kext, double *emis) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  rt_cell(c, ncomp, nlam, comp_w, Kabs_c, Ksca_c, BB, T[c], l1, l2, w1, w2, &kext[c], &emis[c]);
}

__global__ void rt_ray_kernel(const __grid_constant__ TModel m, const double *dens, const double *kext,
                              const double *emis, int nr, int nphi, const double *Rimg, const double *phi,
                              double angle, double fstar, double dimstar, int tracestar, double *image,
                              unsigned int *bad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nr * nphi) return;
  const int i = t / nphi, k = t % nphi;
  int steps;
  image[t] = rt_ray(m, dens, kext, emis, Rimg[i], phi[k], angle, fstar, dimstar, tracestar, RT_MAXSTEPS, &steps);
  if (steps < 0) atomicAdd(bad, 1u);
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

struct RtMem {
  std::vector<void *> p;
  ~RtMem() {
    for (void *q : p) cudaFree(q);
  }
  template <class T>
  cudaError_t alloc(T **out, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (n ? n : 1));
    if (e == cudaSuccess) p.push_back(q);
    *out = (T *)q;
    return e;
  }
};

struct RtDeviceBackend {
  mcg_ctx *ctx = nullptr;
  cudaStream_t st = nullptr;
  RtMem *mem = nullptr;
  TModel tm;
  const double *T = nullptr;
  double *kext = nullptr, *emis = nullptr, *dRimg = nullptr, *dphi = nullptr, *dimage = nullptr;
  unsigned int *dbad = nullptr;
  size_t nimage = 0;
  const double *lam = nullptr; /* host copy */
  int nlam = 0;
  std::string err;

  bool fail(cudaError_t e, const char *what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  }
  bool cells(double lam0, double *kext_out, double *emis_out) {
    const DevModel &m = ctx->model;
    int l1, l2;
    double w1, w2;
    rt_lam(nlam, lam, lam0, &l1, &l2, &w1, &w2);
    rt_cell_kernel<<<nblk(m.ncell, 256), 256, 0, st>>>(m.ncell, m.ncomp, m.nlam, m.comp_w, m.Kabs_c, m.Ksca_c, m.BB,
                                                       T, l1, l2, w1, w2, kext, emis);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(kext_out, kext, sizeof(double) * m.ncell, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(emis_out, emis, sizeof(double) * m.ncell, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? true : fail(e, "trace: cell kernel");
  }
  bool rays(const std::vector<double> &R, const std::vector<double> &phi, double fstar, const RtOptions &o,
            double *image, int *bad) {
    const int nr = (int)R.size(), nphi = (int)phi.size();
    const size_t n = (size_t)nr * nphi;
    cudaError_t e = cudaSuccess;
    if (n > nimage) {
      if ((e = mem->alloc(&dimage, n)) != cudaSuccess) return fail(e, "trace: allocation");
      nimage = n;
    }
    if (!dRimg) {
      if ((e = mem->alloc(&dRimg, (size_t)nr)) != cudaSuccess || (e = mem->alloc(&dphi, (size_t)nphi)) != cudaSuccess ||
          (e = mem->alloc(&dbad, 1)) != cudaSuccess)
        return fail(e, "trace: allocation");
      e = cudaMemcpyAsync(dRimg, R.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dphi, phi.data(), sizeof(double) * nphi, cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return fail(e, "trace: upload");
    }
    e = cudaMemsetAsync(dbad, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return fail(e, "trace: memset");
    rt_ray_kernel<<<nblk((long long)n, 128), 128, 0, st>>>(tm, ctx->model.dens, kext, emis, nr, nphi, dRimg, dphi,
                                                           o.angle, fstar, o.dimstar, o.tracestar, dimage, dbad);
    unsigned int hb = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(image, dimage, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, dbad, sizeof(unsigned int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "trace: ray kernel");
    *bad = (int)hb;
    return true;
  }
};

}  // namespace

mcg_status mcg_trace_spectrum_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, int32_t nobs,
                                   const double *lam_obs, double *flux, int32_t *info) {
  DevModel &m = ctx->model;
  if (!m.valid) return mcg_fail(ctx, MCG_ERR_STATE, "trace_spectrum: no model set");
  if (!o || !T || (nobs > 0 && (!lam_obs || !flux)) || nobs < 0)
    return mcg_fail(ctx, MCG_ERR_ARG, "trace_spectrum: missing argument");
  if (o->nphi < 1 || o->nr == 0 || o->nphi > 100000 || (o->nRfix > 0 && !o->Rfix) || o->nRfix < 0 ||
      !(o->lam_path > 0.0))
    return mcg_fail(ctx, MCG_ERR_ARG, "trace_spectrum: nphi >= 1, nr != 0, lam_path > 0 required");
  const int ncell = m.ncell;
  for (int c = 0; c < ncell; ++c)
    if (!(T[c] >= 0.0) || !(T[c] < 1e6)) return mcg_fail(ctx, MCG_ERR_ARG, "trace_spectrum: T[%d] = %g", c, T[c]);
  cudaStream_t st = ctx->stream;
  std::vector<double> R(m.nr + 1), Theta(m.nt), dens(ncell), lam(m.nlam), Fstar(m.nlam);
  MCG_CUDA(ctx, cudaMemcpyAsync(R.data(), m.R, sizeof(double) * R.size(), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(Theta.data(), m.Theta, sizeof(double) * Theta.size(), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(dens.data(), m.dens, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  if (m.lam_h.size() != (size_t)m.nlam || m.Fstar_h.size() != (size_t)m.nlam)
    return mcg_fail(ctx, MCG_ERR_STATE, "trace_spectrum: the model's wavelengths are not kept");
  lam = m.lam_h;
  Fstar = m.Fstar_h;
  RtMem mem;
  RtDeviceBackend be;
  be.ctx = ctx;
  be.st = st;
  be.mem = &mem;
  be.lam = lam.data();
  be.nlam = m.nlam;
  double *dT;
  cudaError_t e = mem.alloc(&dT, (size_t)ncell);
  if (e == cudaSuccess) e = mem.alloc(&be.kext, (size_t)ncell);
  if (e == cudaSuccess) e = mem.alloc(&be.emis, (size_t)ncell);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, T, sizeof(double) * ncell, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "trace_spectrum: %s", cudaGetErrorString(e));
  be.T = dT;
  TModel hm;
  memset(&hm, 0, sizeof hm);
  hm.nr = m.nr;
  hm.nt = m.nt;
  hm.nc = m.nc;
  hm.ncell = ncell;
  hm.scat_how = m.scat_how;
  hm.R = R.data();
  hm.Theta = Theta.data();
  be.tm = hm;
  be.tm.R = m.R;
  be.tm.Theta = m.Theta;
  RtOptions ro{o->angle, o->nphi, o->nr, o->nRfix, o->Rfix, o->lam_path, o->tracestar, o->dimstar};
  std::vector<double> Rimg;
  int bad = 0;
  if (!rt_spectrum(hm, be, ro, m.nlam, lam.data(), Fstar.data(), dens.data(), nobs, lam_obs, flux, &Rimg, nullptr,
                   &bad))
    return mcg_fail(ctx, MCG_ERR_CUDA, "%s", be.err.c_str());
  if (info) {
    info[0] = (int32_t)Rimg.size();
    info[1] = bad;
  }
  return MCG_OK;
}
