/*
 * dstruct.cu -- mcg_disk_structure (DiskStructure, DiskStructure.f:85-468)
 * on the device.
 *
 *   ds_column_kernel  one thread per (ring, species) column: the hydrostatic
 *                     ODE march from the midplane up (odeint/rkqs/rkck), the
 *                     fixed-zone profile, or the closed-form profile of a
 *                     grain's other scale-height type (formed on the host),
 *                     then the mass renormalisation
 *   ds_cell_kernel    one thread per cell of rings 1..nR-1: densities and
 *                     abundances from the species' profiles
 *   ds_check_kernel   one thread per cell: CheckCells
 * The column set-up (masses, scale factors, fixed zones) and the geometry
 * tables are host logic shared with the test replay (dstruct_core.cuh).
 */
#include <cuda_runtime.h>

#include <vector>

#include "dstruct_core.cuh"
#include "mcg_internal.h"

namespace {

struct DsDev {
  int nc, ncol, nr, ng;
  double Mstar;
  const double *Temp, *V, *R_av, *z, *st, *ct, *cot, *theta_av, *prof;
  const DsColumn *cols;
  const int *ring;
  double *rho;
};

__global__ void ds_column_kernel(const __grid_constant__ DsDev d) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.ncol) return;
  const int i = d.ring[q], nc = d.nc;
  const DsColumn col = d.cols[q];
  ds_column(col, nc, d.R_av[i], d.Mstar, d.Temp + (size_t)i * nc, d.V + (size_t)i * nc, d.z + (size_t)i * nc,
            d.st, d.ct, d.cot, d.theta_av, col.pre >= 0 ? d.prof + col.pre : nullptr, d.rho + (size_t)q * nc);
}

__global__ void ds_cell_kernel(int nr, int nc, int ng, const double *rho, double *dens, double *dens0,
                               double *gasdens, double *w, double *w0) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(nr - 1) * nc) return;
  const int i = 1 + (int)(t / nc), j = (int)(t % nc);
  const size_t c = (size_t)i * nc + j, ns = (size_t)ng + 1;
  ds_cell(ng, rho + (size_t)(i - 1) * ns * nc + j, (size_t)nc, &dens[c], &dens0[c], &gasdens[c], &w[c * ng],
          &w0[c * ng]);
}

__global__ void ds_check_kernel(long long ncell, int ng, double *dens, const double *dens0, double *w,
                                const double *w0) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  ds_check_cell(ng, &dens[c], dens0[c], &w[(size_t)c * ng], &w0[(size_t)c * ng]);
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

/* device memory of one call, freed on every path */
struct DsMem {
  std::vector<void *> p;
  ~DsMem() {
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

struct DsDeviceBackend {
  cudaStream_t st = nullptr;
  /* device copies of the cell arrays, uploaded before the call */
  double *dens = nullptr, *dens0 = nullptr, *gasdens = nullptr, *w = nullptr, *w0 = nullptr;
  const double *Temp = nullptr, *V = nullptr;
  DsMem *mem = nullptr;
  std::string err;

  bool fail(cudaError_t e, const char *what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  }
  template <class T>
  bool up(T **dst, const T *src, size_t n) {
    cudaError_t e = mem->alloc(dst, n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, st);
    return e == cudaSuccess ? true : fail(e, "disk structure: upload");
  }
  bool columns(const DsGrid &g, const DsTables &t, const double *, int ncol, const DsColumn *cols, const int *ring,
               const std::vector<double> &prof, double *) {
    const int nc = g.nt - 1;
    DsDev d;
    d.nc = nc;
    d.ncol = ncol;
    d.nr = g.nr;
    d.ng = g.ng;
    d.Mstar = g.Mstar;
    d.Temp = Temp;
    d.V = V;
    double *a;
    if (!up(&a, t.R_av.data(), t.R_av.size())) return false;
    d.R_av = a;
    if (!up(&a, t.z.data(), t.z.size())) return false;
    d.z = a;
    if (!up(&a, t.st.data(), t.st.size())) return false;
    d.st = a;
    if (!up(&a, t.ct.data(), t.ct.size())) return false;
    d.ct = a;
    if (!up(&a, t.cot.data(), t.cot.size())) return false;
    d.cot = a;
    if (!up(&a, t.theta_av.data(), t.theta_av.size())) return false;
    d.theta_av = a;
    d.prof = nullptr;
    if (!prof.empty()) {
      if (!up(&a, prof.data(), prof.size())) return false;
      d.prof = a;
    }
    DsColumn *dc;
    int *dr;
    if (!up(&dc, cols, (size_t)ncol)) return false;
    if (!up(&dr, ring, (size_t)ncol)) return false;
    d.cols = dc;
    d.ring = dr;
    cudaError_t e = mem->alloc(&d.rho, (size_t)ncol * nc);
    if (e != cudaSuccess) return fail(e, "disk structure: allocation");
    rho = d.rho;
    ds_column_kernel<<<nblk(ncol, 64), 64, 0, st>>>(d);
    e = cudaGetLastError();
    return e == cudaSuccess ? true : fail(e, "disk structure: column kernel");
  }
  double *rho = nullptr;
  bool cells(const DsGrid &g, const double *, double *, double *, double *, double *, double *) {
    const int nc = g.nt - 1;
    const long long ncell = (long long)g.nr * nc;
    ds_cell_kernel<<<nblk((long long)(g.nr - 1) * nc, 128), 128, 0, st>>>(g.nr, nc, g.ng, rho, dens, dens0, gasdens,
                                                                         w, w0);
    ds_check_kernel<<<nblk(ncell, 128), 128, 0, st>>>(ncell, g.ng, dens, dens0, w, w0);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? true : fail(e, "disk structure: cell kernels");
  }
};

}  // namespace

mcg_status mcg_disk_structure_impl(mcg_ctx *ctx, const mcg_structure *s, const double *Temp, double *dens,
                                   double *dens0, double *gasdens, double *w, double *w0) {
  if (!s || !Temp || !dens || !dens0 || !gasdens || !w || !w0 || !s->R || !s->Theta || !s->V)
    return mcg_fail(ctx, MCG_ERR_ARG, "disk_structure: missing array");
  if (s->nr < 2 || s->nt < 3 || s->ngrains < 1 || (s->nzones > 0 && !s->zones) || !(s->Mstar > 0.0))
    return mcg_fail(ctx, MCG_ERR_ARG, "disk_structure: nr >= 2, nt >= 3, ngrains >= 1, Mstar > 0 required");
  const int nc = s->nt - 1, ng = s->ngrains;
  if (s->shtype)
    for (int k = 0; k < ng; ++k)
      if (s->shtype[k] < 0 || s->shtype[k] >= DS_SH_NTYPES)
        return mcg_fail(ctx, MCG_ERR_ARG, "disk_structure: shtype[%d] = %d is not a scale-height type", k,
                        (int)s->shtype[k]);
  const size_t ncell = (size_t)s->nr * nc;
  for (size_t c = 0; c < ncell; ++c)
    if (!(Temp[c] > 0.0)) return mcg_fail(ctx, MCG_ERR_ARG, "disk_structure: Temp[%zu] = %g is not positive", c, Temp[c]);
  std::vector<DsZone> zones(s->nzones > 0 ? s->nzones : 0);
  for (int k = 0; k < s->nzones; ++k) {
    const mcg_zone &z = s->zones[k];
    zones[k] = DsZone{z.rin, z.rout, z.sh, z.rsh, z.shpow, z.denspow, z.fix_struct};
  }
  DsGrid g{s->nr, s->nt, ng, s->R, s->Theta, s->V, s->Mstar, s->nzones, zones.data(), s->shscale, s->grain_scale,
           (const int *)s->shtype};
  cudaStream_t st = ctx->stream;
  DsMem mem;
  DsDeviceBackend be;
  be.st = st;
  be.mem = &mem;
  if (!be.up(&be.dens, dens, ncell) || !be.up(&be.dens0, dens0, ncell) || !be.up(&be.gasdens, gasdens, ncell) ||
      !be.up(&be.w, w, ncell * ng) || !be.up(&be.w0, w0, ncell * ng) || !be.up((double **)&be.Temp, Temp, ncell) ||
      !be.up((double **)&be.V, s->V, ncell))
    return mcg_fail(ctx, MCG_ERR_CUDA, "%s", be.err.c_str());
  if (!ds_disk_structure(g, be, Temp, dens, dens0, gasdens, w, w0))
    return mcg_fail(ctx, MCG_ERR_CUDA, "%s", be.err.c_str());
  MCG_CUDA(ctx, cudaMemcpyAsync(dens, be.dens, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(dens0, be.dens0, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(gasdens, be.gasdens, sizeof(double) * ncell, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(w, be.w, sizeof(double) * ncell * ng, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaMemcpyAsync(w0, be.w0, sizeof(double) * ncell * ng, cudaMemcpyDeviceToHost, st));
  MCG_CUDA(ctx, cudaStreamSynchronize(st));
  return MCG_OK;
}
