/*
 * mcg_api.cu -- the extern "C" entry points of libmcmax_gpu (declared in
 * include/mcmax_gpu.h): context management, error reporting and argument
 * checks in front of the kernel translation units.
 */
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <new>

#include "mcg_internal.h"

mcg_status mcg_fail(mcg_ctx *ctx, mcg_status st, const char *fmt, ...) {
  if (ctx) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return st;
}

extern "C" {

int mcg_version(void) { return 100; }

mcg_status mcg_create(mcg_ctx **out, int device) {
  if (!out) return MCG_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return MCG_ERR_CUDA;
  if (device < 0 || device >= n) return MCG_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return MCG_ERR_CUDA;
  mcg_ctx *c = new (std::nothrow) mcg_ctx();
  if (!c) return MCG_ERR_NOMEM;
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    delete c;
    return MCG_ERR_CUDA;
  }
  c->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return MCG_ERR_CUDA;
  }
  *out = c;
  return MCG_OK;
}

void mcg_destroy(mcg_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  mcg_free_model(ctx->model);
  mcg_free_run(ctx->run);
  if (ctx->part_scratch.p) cudaFree(ctx->part_scratch.p);
  mcg_free_mlp(ctx);
  mcg_free_batch(ctx);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *mcg_last_error(const mcg_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

mcg_status mcg_compute_part(mcg_ctx *ctx, const mcg_part_in *in, mcg_part_out *out) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_part_batch_impl(ctx, 1, in, out);
}

mcg_status mcg_compute_part_batch(mcg_ctx *ctx, int nparts, const mcg_part_in *in, mcg_part_out *out) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_part_batch_impl(ctx, nparts, in, out);
}

mcg_status mcg_compute_part_static(mcg_ctx *ctx, const mcg_part_in *in, mcg_part_out *out) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_part_static_impl(ctx, in, out);
}

mcg_status mcg_set_model(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_set_model_impl(ctx, grid, opac);
}

mcg_status mcg_mcradiation(mcg_ctx *ctx, const mcg_run *run, int64_t *nphot_inout, mcg_result *res) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_mcradiation_impl(ctx, run, nphot_inout, res);
}

mcg_status mcg_add_model(mcg_ctx *ctx, const mcg_grid *grid, const mcg_opacity *opac, int *model_id) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_add_model_impl(ctx, grid, opac, model_id);
}

mcg_status mcg_mcradiation_batch(mcg_ctx *ctx, int nmodels, const int *model_ids, const mcg_run *runs,
                                 int64_t *nphot_inout, mcg_result *results, mcg_batch_opts *opts) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_batch_impl(ctx, nmodels, model_ids, runs, nphot_inout, results, opts);
}

mcg_status mcg_finalize_t(mcg_ctx *ctx, double *T, double *dT, double *dEJv) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_finalize_impl(ctx, T, dT, dEJv);
}

mcg_status mcg_trace_spectrum(mcg_ctx *ctx, const mcg_trace_opts *opts, const double *T, int32_t nobs,
                              const double *lam_obs, double *flux, int32_t *info) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_trace_spectrum_impl(ctx, opts, T, nobs, lam_obs, flux, info);
}

mcg_status mcg_scatter_field(mcg_ctx *ctx, const mcg_trace_opts *opts, const double *T, double lam0, double *field,
                             int64_t cap, int64_t *info) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_scatter_field_impl(ctx, opts, T, lam0, field, cap, info);
}

mcg_status mcg_trace_image(mcg_ctx *ctx, const mcg_trace_opts *opts, const double *T, double lam0,
                           const mcg_image_opts *io, double *flux, double *im, int32_t *info) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_trace_image_impl(ctx, opts, T, lam0, io, flux, im, info);
}

mcg_status mcg_disk_structure(mcg_ctx *ctx, const mcg_structure *s, const double *Temp, double *dens, double *dens0,
                              double *gasdens, double *w, double *w0) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_disk_structure_impl(ctx, s, Temp, dens, dens0, gasdens, w, w0);
}

mcg_status mcg_diffuse(mcg_ctx *ctx, int32_t nphotmin, double dtmax, double factRW, const int32_t *Ni,
                       const double *dT, double *T, double *EJv, int32_t *ncells) {
  if (!ctx) return MCG_ERR_ARG;
  cudaSetDevice(ctx->device);
  return mcg_diffuse_impl(ctx, nphotmin, dtmax, factRW, Ni, dT, T, EJv, ncells);
}

}  // extern "C"
