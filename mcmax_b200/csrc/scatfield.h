/*
 * scatfield.h -- the scattered-light field of the ray tracer on the device
 * (scatfield.cu), used by raytrace.cu.
 */
#ifndef MCMAX_SCATFIELD_H
#define MCMAX_SCATFIELD_H

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "mcg_internal.h"
#include "scat_core.cuh"

/* the field's Monte Carlo settings (an observation's Nphot, NphotAngle and
 * nexits, Telescope.f:606-619) */
struct SfOpts {
  long long nphot;  /* TraceMono packets of one field */
  long long nstar;  /* MakeStarScatter packets */
  uint64_t seed;    /* Philox key of the first field; each later field of a call takes the next key */
  int nexits;       /* EmissionDistribution exit rays per cell (0: none) */
};

/* device state of the fields of one mcg_trace_* call */
struct SfState {
  mcg_ctx *ctx = nullptr;
  cudaStream_t st = nullptr;
  int mode = 0;           /* 0 none, 1 isotropic (one field per grid wavelength), 2 angular (one per wavelength) */
  SfOpts o{};
  double angle = 0.0;
  SfGeomHost gh;
  SfGeom g{};             /* device pointers */
  double *thet = nullptr; /* nt polar edges */
  double *kabs = nullptr, *kext = nullptr, *ksca = nullptr, *albedo = nullptr, *F = nullptr;
  double *emis = nullptr, *vis = nullptr, *cum = nullptr, *dirs = nullptr;
  unsigned long long *stats = nullptr; /* [0] geometry failures, [1] interaction cap, [2] emission retries */
  size_t field_len = 0;   /* doubles of one field */
  std::map<int, double *> iso; /* mode 1: field per grid wavelength */
  double *field = nullptr;     /* mode 2: the field of the last wavelength */
  unsigned long long nfields = 0;
  std::vector<void *> owned;
  std::string err;

  ~SfState();
  bool fail(cudaError_t e, const char *what);
  template <class T>
  bool alloc(T **p, size_t n);
  /* mode from the model: scat_how 2 -> 2, 1 -> 1, else 0 (and 0 when both
   * packet counts are 0 or nothing scatters); allocates and uploads the
   * sub-cell tables and the observer directions of the inclination */
  bool init(mcg_ctx *c, double angle, const SfOpts &opts, const double *Theta_h);
  /* the field of one TraceMono call at wavelength lam0 into out (device,
   * field_len doubles), T the device temperatures */
  bool compute(double lam0, const double *T, double *out);
  /* the per-cell albedo at lam0 into the albedo buffer (TraceFlux's
   * C%Albedo) */
  bool albedo_at(double lam0);
  /* the field(s) a ray pass at lam0 reads: mode 2 the field at lam0, mode 1
   * the fields of the grid wavelengths around it (cached) */
  bool prepare(double lam0, const double *T, const double **f1, const double **f2, double *w1, double *w2);
};

#endif /* MCMAX_SCATFIELD_H */
