/*
 * raytrace.cu -- mcg_trace_spectrum: the ray-traced flux of the current
 * model at one inclination (rt_core.cuh for the algorithm and its
 * reference lines).
 *
 *   rt_cell_kernel  one thread per cell: extinction and source function at
 *                   a wavelength
 *   rt_ray_kernel   one thread per image ray (radius, angle): the path
 *                   through the cells and the formal solution, with the
 *                   scattered light of the field of scatfield.cu when the
 *                   options ask for one
 * The image grid, the tau = 0.1 radius and the flux sum are host logic
 * shared with the test replay.
 *
 * mcg_trace_image adds the rectangular image of one wavelength:
 *   rt_image_sample_kernel  one thread per sample point: the interpolated
 *                           intensity and the pixels of the point and its
 *                           mirror (rt_image_sample)
 *   stable radix sort of (pixel, amount) pairs, in sample order
 *   rt_image_add_kernel     one thread per pixel: adds its run of amounts in
 *                           sample order, so that every pixel holds the same
 *                           sum, bit for bit, as the sequential loop
 * The samples are processed in chunks of RT_IMG_CHUNK; the pixel sums carry
 * over from chunk to chunk.
 */
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <vector>

#include "mcg_internal.h"
#include "rt_core.cuh"
#include "scatfield.h"

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
                              unsigned int *bad, const __grid_constant__ RtScat sc, int has_sc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nr * nphi) return;
  const int i = t / nphi, k = t % nphi;
  int steps;
  image[t] = rt_ray(m, dens, kext, emis, Rimg[i], phi[k], angle, fstar, dimstar, tracestar, RT_MAXSTEPS, &steps,
                    has_sc ? &sc : nullptr);
  if (steps < 0) atomicAdd(bad, 1u);
}

__global__ void rt_image_sample_kernel(long long s0, long long n, int nphi, int nint, const double *R,
                                       const double *image, unsigned long long seed, double Rmax, double pa_deg,
                                       int npix, int linear, uint32_t *keys, double *vals) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t key[2];
  double v;
  rt_image_sample(s0 + t, nphi, nint, R, image, (uint64_t)seed, Rmax, pa_deg, npix, linear, key, &v);
  keys[2 * t] = key[0];
  keys[2 * t + 1] = key[1];
  vals[2 * t] = v;
  vals[2 * t + 1] = v;
}

/* first index q in [0, n) with keys[q] >= p (n when none) */
__device__ __forceinline__ long long rt_lower_bound(const uint32_t *keys, long long n, uint32_t p) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (keys[mid] < p)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void rt_image_add_kernel(int npix2, long long n, const uint32_t *keys, const double *vals, double *im) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix2) return;
  const long long lo = rt_lower_bound(keys, n, (uint32_t)p), hi = rt_lower_bound(keys, n, (uint32_t)p + 1u);
  if (lo == hi) return;
  double a = im[p];
  for (long long q = lo; q < hi; ++q) a = a + vals[q];
  im[p] = a;
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
  SfState *sf = nullptr;       /* the scattered-light fields, or null */
  RtScat sc{};
  int has_sc = 0;
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
  bool field(double lam0) {
    has_sc = 0;
    if (!sf || !sf->mode) return true;
    const double *f1, *f2;
    double w1, w2;
    if (!sf->prepare(lam0, T, &f1, &f2, &w1, &w2)) {
      err = sf->err;
      return false;
    }
    sc.mode = sf->mode;
    sc.g = sf->g;
    sc.thet = sf->thet;
    sc.f1 = f1;
    sc.f2 = f2;
    sc.w1 = w1;
    sc.w2 = w2;
    sc.albedo = sf->albedo;
    sc.V = ctx->model.V;
    has_sc = 1;
    return true;
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
                                                           o.angle, fstar, o.dimstar, o.tracestar, dimage, dbad, sc,
                                                           has_sc);
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

/* the ray-traced flux at nobs wavelengths (shared by both entry points):
 * validation, the image rays and the formal solution; Rimg and image_last
 * receive the image radii and the last wavelength's intensities */
static mcg_status rt_trace(mcg_ctx *ctx, const char *who, const mcg_trace_opts *o, const double *T, int32_t nobs,
                           const double *lam_obs, double *flux, std::vector<double> *Rimg,
                           std::vector<double> *image_last, int *bad) {
  DevModel &m = ctx->model;
  if (!m.valid) return mcg_fail(ctx, MCG_ERR_STATE, "%s: no model set", who);
  if (!o || !T || (nobs > 0 && (!lam_obs || !flux)) || nobs < 0)
    return mcg_fail(ctx, MCG_ERR_ARG, "%s: missing argument", who);
  if (o->nphi < 1 || o->nr == 0 || o->nphi > 100000 || (o->nRfix > 0 && !o->Rfix) || o->nRfix < 0 ||
      !(o->lam_path > 0.0))
    return mcg_fail(ctx, MCG_ERR_ARG, "%s: nphi >= 1, nr != 0, lam_path > 0 required", who);
  if (o->nphot_scatter < 0 || o->nphot_star < 0 || o->nphot_scatter > 2000000000LL || o->nphot_star > 2000000000LL ||
      o->nexits < 0 || o->nexits == 1 || o->nexits > 10000)
    return mcg_fail(ctx, MCG_ERR_ARG, "%s: 0 <= nphot_scatter, nphot_star <= 2e9 and nexits 0 or 2..10000 required",
                    who);
  const int ncell = m.ncell;
  for (int c = 0; c < ncell; ++c)
    if (!(T[c] >= 0.0) || !(T[c] < 1e6)) return mcg_fail(ctx, MCG_ERR_ARG, "%s: T[%d] = %g", who, c, T[c]);
  cudaStream_t st = ctx->stream;
  std::vector<double> R(m.nr + 1), Theta(m.nt), dens(ncell), lam(m.nlam), Fstar(m.nlam);
  MCG_CUDA(ctx, cudaMemcpyAsync(R.data(), m.R, sizeof(double) * R.size(), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(Theta.data(), m.Theta, sizeof(double) * Theta.size(), cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(dens.data(), m.dens, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  if (m.lam_h.size() != (size_t)m.nlam || m.Fstar_h.size() != (size_t)m.nlam)
    return mcg_fail(ctx, MCG_ERR_STATE, "%s: the model's wavelengths are not kept", who);
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
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
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
  SfState sf;
  if (o->nphot_scatter > 0 || o->nphot_star > 0) {
    SfOpts so{(long long)o->nphot_scatter, (long long)o->nphot_star, o->seed_scatter, o->nexits};
    if (!sf.init(ctx, o->angle, so, Theta.data())) return mcg_fail(ctx, MCG_ERR_CUDA, "%s: %s", who, sf.err.c_str());
    be.sf = &sf;
  }
  *bad = 0;
  if (!rt_spectrum(hm, be, ro, m.nlam, lam.data(), Fstar.data(), dens.data(), nobs, lam_obs, flux, Rimg, image_last,
                   bad))
    return mcg_fail(ctx, MCG_ERR_CUDA, "%s", be.err.c_str());
  return MCG_OK;
}

mcg_status mcg_trace_spectrum_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, int32_t nobs,
                                   const double *lam_obs, double *flux, int32_t *info) {
  std::vector<double> Rimg;
  int bad = 0;
  const mcg_status rc = rt_trace(ctx, "trace_spectrum", o, T, nobs, lam_obs, flux, &Rimg, nullptr, &bad);
  if (rc != MCG_OK) return rc;
  if (info) {
    info[0] = (int32_t)Rimg.size();
    info[1] = bad;
  }
  return MCG_OK;
}

constexpr long long RT_IMG_CHUNK = 1LL << 23; /* samples per sort (2^24 pairs, 192 MB with the sort buffers) */

mcg_status mcg_trace_image_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, double lam0,
                                const mcg_image_opts *io, double *flux, double *im, int32_t *info) {
  if (!io || !im || !flux) return mcg_fail(ctx, MCG_ERR_ARG, "trace_image: missing argument");
  if (io->npixel < 1 || io->npixel > 8192 || io->nint < 1 || io->nint > 1000000 || !(io->Rmax > 0.0) ||
      !(io->Rmax < 1e30) || !(fabs(io->pa) < 1e6) || io->cap < 0 || (io->cap > 0 && (!io->Rimg || !io->rphi)))
    return mcg_fail(ctx, MCG_ERR_ARG,
                    "trace_image: 1 <= npixel <= 8192, 1 <= nint <= 1e6, 0 < Rmax < 1e30, |pa| < 1e6 and the "
                    "radius buffers required");
  std::vector<double> Rimg, rphi;
  int bad = 0;
  mcg_status rc = rt_trace(ctx, "trace_image", o, T, 1, &lam0, flux, &Rimg, &rphi, &bad);
  if (rc != MCG_OK) return rc;
  const int nr = (int)Rimg.size(), nphi = o->nphi, npix = io->npixel;
  if (info) {
    info[0] = nr;
    info[1] = bad;
  }
  if (io->cap > 0) {
    if (io->cap < nr) return mcg_fail(ctx, MCG_ERR_ARG, "trace_image: cap %d < %d image radii", io->cap, nr);
    memcpy(io->Rimg, Rimg.data(), sizeof(double) * nr);
    memcpy(io->rphi, rphi.data(), sizeof(double) * (size_t)nr * nphi);
  }
  const int npix2 = npix * npix;
  const long long nsamp = (long long)(nr - 1) * nphi * io->nint;
  const long long chunk = nsamp < RT_IMG_CHUNK ? nsamp : RT_IMG_CHUNK;
  cudaStream_t st = ctx->stream;
  RtMem mem;
  double *dR, *dI, *dim, *vals, *vals_s;
  uint32_t *keys, *keys_s;
  cudaError_t e = mem.alloc(&dR, (size_t)nr);
  if (e == cudaSuccess) e = mem.alloc(&dI, (size_t)nr * nphi);
  if (e == cudaSuccess) e = mem.alloc(&dim, (size_t)npix2);
  if (e == cudaSuccess) e = mem.alloc(&keys, (size_t)(2 * chunk));
  if (e == cudaSuccess) e = mem.alloc(&keys_s, (size_t)(2 * chunk));
  if (e == cudaSuccess) e = mem.alloc(&vals, (size_t)(2 * chunk));
  if (e == cudaSuccess) e = mem.alloc(&vals_s, (size_t)(2 * chunk));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dR, Rimg.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dI, rphi.data(), sizeof(double) * (size_t)nr * nphi, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dim, 0, sizeof(double) * npix2, st);
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "trace_image: %s", cudaGetErrorString(e));
  int end_bit = 1;
  while (end_bit < 32 && (1ull << end_bit) <= (unsigned long long)npix2) ++end_bit; /* keys 0..npix2 */
  size_t tmp_bytes = 0;
  e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys_s, vals, vals_s, (int)(2 * chunk), 0, end_bit,
                                      st);
  char *tmp = nullptr;
  if (e == cudaSuccess) e = mem.alloc(&tmp, tmp_bytes);
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "trace_image: sort setup: %s", cudaGetErrorString(e));
  for (long long s0 = 0; s0 < nsamp; s0 += chunk) {
    const long long n = nsamp - s0 < chunk ? nsamp - s0 : chunk;
    rt_image_sample_kernel<<<nblk(n, 256), 256, 0, st>>>(s0, n, nphi, io->nint, dR, dI,
                                                         (unsigned long long)io->seed, io->Rmax, io->pa, npix,
                                                         io->linear ? 1 : 0, keys, vals);
    e = cudaGetLastError();
    size_t need = 0;
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_s, vals, vals_s, (int)(2 * n), 0, end_bit, st);
    if (e == cudaSuccess && need > tmp_bytes)
      return mcg_fail(ctx, MCG_ERR_CUDA, "trace_image: sort needs %zu bytes, %zu held", need, tmp_bytes);
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys_s, vals, vals_s, (int)(2 * n), 0, end_bit, st);
    if (e == cudaSuccess) {
      rt_image_add_kernel<<<nblk(npix2, 256), 256, 0, st>>>(npix2, 2 * n, keys_s, vals_s, dim);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "trace_image: image pass: %s", cudaGetErrorString(e));
  }
  MCG_CUDA(ctx, cudaMemcpyAsync(im, dim, sizeof(double) * npix2, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  return MCG_OK;
}

mcg_status mcg_scatter_field_impl(mcg_ctx *ctx, const mcg_trace_opts *o, const double *T, double lam0, double *field,
                                  int64_t cap, int64_t *info) {
  DevModel &m = ctx->model;
  if (!m.valid) return mcg_fail(ctx, MCG_ERR_STATE, "scatter_field: no model set");
  if (!o || !T || !info || cap < 0) return mcg_fail(ctx, MCG_ERR_ARG, "scatter_field: missing argument");
  if (o->nphot_scatter < 0 || o->nphot_star < 0 || o->nphot_scatter > 2000000000LL || o->nphot_star > 2000000000LL ||
      o->nexits < 0 || o->nexits == 1 || o->nexits > 10000 || !(lam0 > 0.0))
    return mcg_fail(ctx, MCG_ERR_ARG, "scatter_field: packet counts 0..2e9, nexits 0 or 2..10000, lam0 > 0");
  const int ncell = m.ncell;
  for (int c = 0; c < ncell; ++c)
    if (!(T[c] >= 0.0) || !(T[c] < 1e6)) return mcg_fail(ctx, MCG_ERR_ARG, "scatter_field: T[%d] = %g", c, T[c]);
  cudaStream_t st = ctx->stream;
  std::vector<double> Theta(m.nt);
  MCG_CUDA(ctx, cudaMemcpyAsync(Theta.data(), m.Theta, sizeof(double) * m.nt, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  SfState sf;
  SfOpts so{(long long)o->nphot_scatter, (long long)o->nphot_star, o->seed_scatter, o->nexits};
  if (!sf.init(ctx, o->angle, so, Theta.data())) return mcg_fail(ctx, MCG_ERR_CUDA, "scatter_field: %s", sf.err.c_str());
  for (int k = 0; k < 6; ++k) info[k] = 0;
  info[5] = sf.mode;
  if (!sf.mode) return MCG_OK;
  info[0] = sf.gh.nsub;
  info[1] = (int64_t)sf.field_len;
  if (!field) return MCG_OK;
  if (cap < (int64_t)sf.field_len)
    return mcg_fail(ctx, MCG_ERR_ARG, "scatter_field: cap %lld < %zu", (long long)cap, sf.field_len);
  RtMem mem;
  double *dT, *dF;
  cudaError_t e = mem.alloc(&dT, (size_t)ncell);
  if (e == cudaSuccess) e = mem.alloc(&dF, sf.field_len);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, T, sizeof(double) * ncell, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return mcg_fail(ctx, MCG_ERR_CUDA, "scatter_field: %s", cudaGetErrorString(e));
  if (!sf.compute(lam0, dT, dF)) return mcg_fail(ctx, MCG_ERR_CUDA, "%s", sf.err.c_str());
  unsigned long long hs[3] = {0, 0, 0};
  MCG_CUDA(ctx, cudaMemcpyAsync(field, dF, sizeof(double) * sf.field_len, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(hs, sf.stats, sizeof hs, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  info[2] = (int64_t)hs[0];
  info[3] = (int64_t)hs[1];
  info[4] = (int64_t)hs[2];
  return MCG_OK;
}
