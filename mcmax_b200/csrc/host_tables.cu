/*
 * host_tables.cu -- host-side builders of the Planck table the packet loop
 * reads (Init.f:2616-2622 with Planck from Subroutines.f:4-21).
 *
 * The reference evaluates exp(h nu / k T) - 1 in quad precision (real*16) to
 * avoid cancellation at long wavelengths; this keeps that (libquadmath
 * __float128), which the device cannot do, so the table is built on the
 * host, in parallel over wavelengths, and uploaded with the model.
 */
#include <quadmath.h>

#include <cmath>
#include <thread>
#include <vector>

#include "mcg_internal.h"

static double planck_q(double T, double lam) {
  const double k = 1.3807e-16, c = 2.9979e10, h = 6.6261e-27;
  double nu = c / (lam * 1e-4);
  double xd = (h * nu) / (k * T);
  __float128 x = (__float128)xd;
  if (x > (__float128)1e3) return 0.0;
  double num = ((2.0 * h) * ((nu * nu) * nu)) / (c * c);
  __float128 den = expq(x) - (__float128)1.0;
  return (double)((__float128)num / den);
}

extern "C" mcg_status mcg_bb_table(int nlam, const double *lam, double *BB) {
  if (nlam < 1 || !lam || !BB) return MCG_ERR_ARG;
  for (int i = 0; i < nlam; ++i)
    if (!(lam[i] > 0.0)) return MCG_ERR_ARG;
  unsigned nt = std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  if ((int)nt > nlam) nt = (unsigned)nlam;
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([=]() {
      for (int i = (int)t; i < nlam; i += (int)nt) {
        BB[(size_t)i * MCG_TT] = 0.0;
        for (int j = 1; j <= MCG_TMAX; ++j) BB[(size_t)i * MCG_TT + j] = planck_q((double)j, lam[i]);
      }
    });
  for (auto &x : th) x.join();
  return MCG_OK;
}

extern "C" double mcg_planck(double T, double lam) { return planck_q(T, lam); }
