/*
 * part_kernels.cu -- the DHS/Mie opacity stage (ComputePart.f:1-552) on
 * sm_100a.
 *
 * Decomposition of one batch of grain bins ("parts"):
 *   host   : the per-part set-up of ComputePart.f:1-297 (abundance
 *            normalisation, Bruggeman blend with vacuum, Gauss-Legendre
 *            filling fractions, size grid and number weights), producing one
 *            sample per (part, wavelength, material, size, filling fraction).
 *   K1a    : dhs_kernel   -- one warp per coated-sphere sample (dhs_core.cuh);
 *            writes the 4 x 180 Mueller elements and the cross sections of
 *            the sample, or flags Err = 1.
 *   K1b    : mie_kernel   -- one warp per (part, wavelength, material, size)
 *            that needs the homogeneous-sphere fallback (f = 0, x > 1e4, or a
 *            DHS failure, ComputePart.f:332-383).
 *   K1c    : accum_kernel -- one warp per (part, wavelength): replays the
 *            (material, size, f) loop of the reference in its order
 *            (sticky Err, Mie reuse, forward-peak renormalisation
 *            ComputePart.f:407-415, weighted sums :417-429) and writes
 *            Kabs/Ksca/Kext and the six normalised Mueller elements.
 * All FP64, compiled with --fmad=false: the result is bit-identical to the
 * CPU oracle.  Scratch (down-recurrence arrays) lives in one device buffer
 * sliced per resident warp.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dhs_core.cuh"
#include "mcg_internal.h"

namespace {

constexpr int NA = 180;
constexpr int WARP = 32;
constexpr int APL_DHS = 3;  /* ceil(90/32) angles per lane */
constexpr int APL_MIE = 3;

/* status of a sample */
enum : int8_t { S_DHS = 0, S_DHS_ERR = 1, S_MIE = 2 };

struct SampleDev {
  const double *rcore, *rshell, *wvno, *mre, *mim;
  int8_t *status;
  double *F;      /* nsamp*4*180 */
  double *cs;     /* nsamp*2 (cemie, csmie) */
  int *mie_need;  /* per (part, lam, l, k) */
  int nsamp;
};

__global__ void __launch_bounds__(128) dhs_kernel(SampleDev s, const double *mu, cx *scratch,
                                                  int cap, unsigned long long *next) {
  const int lane = threadIdx.x & 31;
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  cx *my = scratch + (size_t)warp_global * 4 * cap;
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(next, 1ULL);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= (unsigned long long)s.nsamp) break;
    const int i = (int)idx;
    if (s.status[i] != S_DHS) continue;
    double *F = s.F + (size_t)i * 4 * NA;
    double ce = 0.0, cs = 0.0;
    int e = dhs_sample<WARP, APL_DHS>(s.rcore[i], s.rshell[i], s.wvno[i], s.mre[i], -s.mim[i], mu,
                                      my, cap, lane, F, F + NA, F + 2 * NA, F + 3 * NA, &ce, &cs);
    if (lane == 0) {
      if (e) {
        s.status[i] = S_DHS_ERR;
      } else {
        s.cs[2 * i] = ce;
        s.cs[2 * i + 1] = cs;
      }
    }
    __syncwarp();
  }
}

struct MieDev {
  const double *rad, *lam, *e1, *e2; /* per mie slot */
  const int *need;
  double *F;   /* nslot*4*180 */
  double *cs;  /* nslot*2 (cemie, csmie) */
  int8_t *ok;
  int nslot;
};

__global__ void __launch_bounds__(128) mie_kernel(MieDev m, double *scratch, int cap,
                                                  unsigned long long *next) {
  const int lane = threadIdx.x & 31;
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double *my = scratch + (size_t)warp_global * 8 * cap;
  for (;;) {
    unsigned long long idx = 0;
    if (lane == 0) idx = atomicAdd(next, 1ULL);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= (unsigned long long)m.nslot) break;
    const int i = (int)idx;
    if (!m.need[i]) continue;
    double *F = m.F + (size_t)i * 4 * NA;
    double cs = 0.0, ce = 0.0;
    int e = mie_sample<WARP, APL_MIE>(m.rad[i], m.lam[i], m.e1[i], m.e2[i], my, cap, lane, F,
                                      F + NA, F + 2 * NA, F + 3 * NA, &cs, &ce);
    if (lane == 0) {
      m.ok[i] = e ? 0 : 1;
      m.cs[2 * i] = ce;
      m.cs[2 * i + 1] = cs;
    }
    __syncwarp();
  }
}

/* per-part description for the accumulation kernel */
struct PartDev {
  int nlam, nmc, ns, nf;
  int samp0;   /* first sample index of the part */
  int mie0;    /* first Mie slot of the part */
  int out0;    /* first output wavelength row of the part */
  double mscale;
  const double *frac;  /* nmc */
  const double *rho;   /* nmc */
  const double *r1;    /* ns */
  const double *nr;    /* nmc*ns */
  const double *wf;    /* nf */
};

struct AccDev {
  const PartDev *parts;
  int nparts;
  const int *row_part;  /* for each output row: part index */
  const int8_t *status;
  const double *sF, *scs;
  const double *mF, *mcs;
  const double *sinw;   /* 180 */
  double tot2;          /* sum of sinw in order */
  double *kabs, *ksca, *kext, *Fout; /* rows x ..., Fout rows*6*180 */
  double *rho_av;       /* per part */
  int nrows;
};

/* ComputePart.f:318-447 for one (part, wavelength), in the reference's loop
 * order.  Lane L owns bins L, L+32, ... of the 180. */
__global__ void __launch_bounds__(128) accum_kernel(AccDev a) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= a.nrows) return;
  const int p = a.row_part[row];
  const PartDev P = a.parts[p];
  const int ilam = row - P.out0;
  constexpr int BPL = (NA + WARP - 1) / WARP; /* 6 */
  double acc[6][BPL];
#pragma unroll
  for (int e = 0; e < 6; ++e)
#pragma unroll
    for (int b = 0; b < BPL; ++b) acc[e][b] = 0.0;
  double csca = 0.0, cabs = 0.0, cext = 0.0, mass = 0.0, vol = 0.0;
  /* Mie working state that survives across f (the reference's Mief arrays) */
  double f11_0 = 0.0;     /* current Mief11(1) */
  for (int l = 0; l < P.nmc; ++l) {
    if (P.frac[l] == 0.0) continue;
    for (int k = 0; k < P.ns; ++k) {
      const double r1 = P.r1[k];
      const int mslot = P.mie0 + (ilam * P.nmc + l) * P.ns + k;
      int err = 0;
      for (int i = 0; i < P.nf; ++i) {
        const int s = P.samp0 + ((ilam * P.nmc + l) * P.ns + k) * P.nf + i;
        const int8_t st = a.status[s];
        if (st == S_DHS_ERR) err = 1;
        const double *src;
        double ce, cs, f22_0;
        if (err || st == S_MIE) {
          src = a.mF + (size_t)mslot * 4 * NA;
          ce = a.mcs[2 * mslot];
          cs = a.mcs[2 * mslot + 1];
          if (err || i == 0) {
            f11_0 = src[0];
          }
          f22_0 = f11_0;  /* Mief22 = Mief11 (current contents) */
        } else {
          src = a.sF + (size_t)s * 4 * NA;
          ce = a.scs[2 * s];
          cs = a.scs[2 * s + 1];
          f11_0 = src[0];
          f22_0 = f11_0;
        }
        /* forward-peak renormalisation, sequential over the 180 bins */
        double t1 = f11_0 * a.sinw[0];
        for (int j = 1; j < NA; ++j) t1 = t1 + src[j] * a.sinw[j];
        f11_0 = f11_0 + (a.tot2 - t1) / a.sinw[0];
        if (f11_0 < 0.0) f11_0 = 0.0;
        const double wn = P.wf[i] * P.nr[l * P.ns + k];
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
          const int j = lane + b * WARP;
          if (j < NA) {
            const double v11 = j == 0 ? f11_0 : src[j];
            const double v22 = j == 0 ? f22_0 : src[j];
            const double v12 = src[NA + j];
            const double v33 = src[2 * NA + j];
            const double v34 = src[3 * NA + j];
            acc[0][b] += (wn * v11) * cs;
            acc[1][b] += (wn * v12) * cs;
            acc[2][b] += (wn * v22) * cs;
            acc[3][b] += (wn * v33) * cs;
            acc[4][b] += (wn * v34) * cs;
            acc[5][b] += (wn * v33) * cs;
          }
        }
        cext = cext + wn * ce;
        csca = csca + wn * cs;
        cabs = cabs + wn * (ce - cs);
        const double r13 = (r1 * r1) * r1;
        mass = mass + (((wn * P.rho[l]) * 4.0) * DHS_PI) * r13 / 3.0;
        vol = vol + ((wn * 4.0) * DHS_PI) * r13 / 3.0;
      }
    }
  }
  if (lane == 0) {
    a.kabs[row] = 1.0e4 * cabs / (mass / P.mscale);
    a.ksca[row] = 1.0e4 * csca / (mass / P.mscale);
    a.kext[row] = 1.0e4 * cext / (mass / P.mscale);
    if (ilam == P.nlam - 1) a.rho_av[p] = mass / vol;
  }
#pragma unroll
  for (int e = 0; e < 6; ++e)
#pragma unroll
    for (int b = 0; b < BPL; ++b) {
      const int j = lane + b * WARP;
      if (j < NA) a.Fout[((size_t)row * 6 + e) * NA + j] = acc[e][b] / csca;
    }
}

/* ---------------- host side ---------------- */

/* Bruggeman mixing, ComputePart.f:1177-1212 (same operation order as the
 * oracle) */
void blender(const double *e1, const double *e2, const double *abun, int nm, double *e1out,
             double *e2out) {
  cx mm = cx_make(1.0, 0.0), me = mm;
  for (int iter = 0; iter < 100; ++iter) {
    cx sum = cx_make(0.0, 0.0);
    cx mm2 = cx_mul(mm, mm);
    for (int j = 0; j < nm; ++j) {
      cx mj = cx_make(e1[j], e2[j]);
      cx mj2 = cx_mul(mj, mj);
      cx q = cx_div(cx_sub(mj2, mm2), cx_add(mj2, cx_scale(2.0, mm2)));
      sum = cx_add(sum, cx_scale(abun[j], q));
    }
    cx num = cx_make(2.0 * sum.re + 1.0, 2.0 * sum.im);
    cx den = cx_make(1.0 - sum.re, -sum.im);
    me = cx_div(num, den);
    me = cx_mul(mm, cx_sqrt(me));
    mm = me;
  }
  *e1out = me.re;
  *e2out = me.im;
}

/* Gauss-Legendre nodes on [x1,x2], ComputePart.f:1219-1249 */
void gauleg2(double x1, double x2, double *x, double *w, int n) {
  int m = (n + 1) / 2;
  double xm = 0.5 * (x2 + x1);
  double xl = 0.5 * (x2 - x1);
  for (int i = 1; i <= m; ++i) {
    double z = cos(3.141592654 * ((double)i - 0.25) / ((double)n + 0.5));
    double z1, pp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= n; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (!(std::fabs(z - z1) > 3.0e-14)) break;
    }
    x[i - 1] = xm - xl * z;
    x[n - i] = xm + xl * z;
    w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

/* per-part host set-up (ComputePart.f:1-297) */
struct PartHost {
  int nlam = 0, nmc = 0, ns = 0, nf = 0;
  double mscale = 1.0, rscale = 1.0;
  std::vector<double> e1, e2;  /* nmc*nlam */
  std::vector<double> frac, rho, f, wf, r, r1, nr;
  std::vector<double> rad, rcore; /* ns*nf */
};

bool part_setup(const mcg_part_in &in, PartHost &h, std::string &why) {
  if (in.nlam < 2 || !in.lam || in.nm < 1 || !in.e1 || !in.e2 || !in.frac || !in.rho) {
    why = "part: nlam >= 2, nm >= 1 and non-null lam/e1/e2/frac/rho are required";
    return false;
  }
  if (!(in.amin > 0.0) || !(in.amax > 0.0) || in.ns < 1 || in.nf < 1) {
    why = "part: amin, amax > 0 and ns, nf >= 1 are required";
    return false;
  }
  if (in.nm + 1 > 64) {
    why = "part: at most 63 materials";
    return false;
  }
  for (int l = 0; l < in.nm; ++l)
    if (!(in.rho[l] > 0.0)) {
      why = "part: material densities must be > 0";
      return false;
    }
  const int nlam = in.nlam, nm = in.nm;
  h.nlam = nlam;
  int nmat = nm + (in.blend ? 1 : 0);
  h.e1.assign(in.e1, in.e1 + (size_t)nm * nlam);
  h.e2.assign(in.e2, in.e2 + (size_t)nm * nlam);
  h.e1.resize((size_t)nmat * nlam);
  h.e2.resize((size_t)nmat * nlam);
  h.frac.resize(nmat);
  h.rho.resize(nmat);
  for (int l = 0; l < nm; ++l) {
    h.rho[l] = in.rho[l];
    h.frac[l] = in.frac[l] / in.rho[l];
  }
  double minlog = log10(in.amin), maxlog = log10(in.amax);
  double pw = -in.apow;
  double maxf = in.fmax;
  int nf = in.nf;
  if (maxf == 0.0) nf = 1;
  double tot = 0.0;
  for (int i = 0; i < nm; ++i) tot += h.frac[i];
  if (in.normalize_abun <= 0.0) {
    for (int i = 0; i < nm; ++i) h.frac[i] /= tot;
    h.mscale = 1.0;
    h.rscale = 1.0;
  } else {
    h.mscale = 0.0;
    for (int i = 0; i < nm; ++i) h.mscale += h.frac[i] * h.rho[i] / in.normalize_abun;
    h.rscale = pow(h.mscale, 1.0 / 3.0);
    for (int i = 0; i < nm; ++i) h.frac[i] /= tot;
  }
  int nmc = nm;
  if (in.blend) {
    nmc = nm + 1;
    for (int i = 0; i < nlam; ++i) {
      h.e1[(size_t)nm * nlam + i] = 1.0;
      h.e2[(size_t)nm * nlam + i] = 0.0;
    }
    h.rho[nm] = 0.0;
    h.frac[nm] = in.porosity;
    for (int l = 0; l < nm; ++l) h.frac[l] *= (1.0 - in.porosity);
    double ee1[64], ee2[64];
    for (int i = 0; i < nlam; ++i) {
      for (int l = 0; l < nmc; ++l) {
        ee1[l] = h.e1[(size_t)l * nlam + i];
        ee2[l] = h.e2[(size_t)l * nlam + i];
      }
      double b1, b2;
      blender(ee1, ee2, h.frac.data(), nmc, &b1, &b2);
      h.e1[i] = b1;
      h.e2[i] = b2;
    }
    double rav = 0.0;
    for (int l = 0; l < nmc; ++l) rav += h.frac[l] * h.rho[l];
    h.rho[0] = rav;
    h.frac[0] = 1.0;
    nmc = 1;
  }
  h.nmc = nmc;
  h.f.assign(nf, 0.0);
  h.wf.assign(nf, 0.0);
  if (nf > 1 && maxf > 0.01) {
    gauleg2(0.01, maxf, h.f.data(), h.wf.data(), nf);
  } else if (maxf == 0.0) {
    for (int i = 0; i < nf; ++i) {
      h.f[i] = 0.0;
      h.wf[i] = 1.0 / (double)nf;
    }
  } else {
    nf = 1;
    h.f.assign(1, maxf);
    h.wf.assign(1, 1.0);
  }
  h.nf = nf;
  const int ns = in.ns;
  h.ns = ns;
  h.r.assign(ns, 0.0);
  h.nr.assign((size_t)nmc * ns, 0.0);
  for (int l = 0; l < nmc; ++l) {
    if (ns == 1) {
      h.r[0] = pow(10.0, (minlog + maxlog) / 2.0);
      h.nr[(size_t)l * ns] = h.frac[l];
    } else {
      double t2 = 0.0;
      for (int k = 0; k < ns; ++k) {
        h.r[k] = pow(10.0, minlog + (maxlog - minlog) * (double)k / (double)(ns - 1));
        h.nr[(size_t)l * ns + k] = pow(h.r[k], pw + 1.0);
        t2 += h.nr[(size_t)l * ns + k] * (h.r[k] * h.r[k] * h.r[k]);
      }
      for (int k = 0; k < ns; ++k) h.nr[(size_t)l * ns + k] = h.frac[l] * h.nr[(size_t)l * ns + k] / t2;
    }
  }
  h.r1.resize(ns);
  h.rad.resize((size_t)ns * nf);
  h.rcore.resize((size_t)ns * nf);
  for (int k = 0; k < ns; ++k) {
    h.r1[k] = h.r[k] * h.rscale;
    for (int i = 0; i < nf; ++i) {
      h.rad[(size_t)k * nf + i] = h.r1[k] / pow(1.0 - h.f[i], 1.0 / 3.0);
      h.rcore[(size_t)k * nf + i] = h.f[i] > 0.0 ? h.rad[(size_t)k * nf + i] * pow(h.f[i], 1.0 / 3.0) : 0.0;
    }
  }
  return true;
}

template <typename T>
T *dev_alloc(std::vector<void *> &own, size_t n, cudaError_t &err) {
  void *p = nullptr;
  if (n == 0) n = 1;
  err = cudaMalloc(&p, n * sizeof(T));
  if (err == cudaSuccess) own.push_back(p);
  return (T *)p;
}

}  // namespace

mcg_status mcg_part_batch_impl(mcg_ctx *ctx, int nparts, const mcg_part_in *in, mcg_part_out *out) {
  if (nparts < 1 || !in || !out) return mcg_fail(ctx, MCG_ERR_ARG, "compute_part: nparts >= 1 and non-null in/out required");
  std::vector<PartHost> H(nparts);
  for (int p = 0; p < nparts; ++p) {
    std::string why;
    if (!part_setup(in[p], H[p], why)) return mcg_fail(ctx, MCG_ERR_ARG, "%s (part %d)", why.c_str(), p);
    if (!out[p].kabs || !out[p].ksca || !out[p].kext || !out[p].F)
      return mcg_fail(ctx, MCG_ERR_ARG, "compute_part: null output array (part %d)", p);
  }
  /* constant tables, ComputePart.f:294-297 and :407-415 */
  double mu[90], sinw[NA], tot2 = 0.0;
  for (int i = 1; i <= 90; ++i) mu[i - 1] = cos(((double)i - 0.5) / (double)(NA / 2) * DHS_PI / 2.0);
  for (int j = 1; j <= NA; ++j) sinw[j - 1] = sin(DHS_PI * ((double)j - 0.5) / (double)NA);
  for (int j = 0; j < NA; ++j) tot2 = tot2 + sinw[j];

  /* enumerate samples and Mie slots */
  std::vector<double> srcore, srshell, swvno, smre, smim;
  std::vector<int8_t> sstat;
  std::vector<double> mrad, mlam, me1, me2;
  std::vector<int> mneed;
  std::vector<PartDev> pd(nparts);
  std::vector<int> row_part;
  int maxnmx1 = 150, maxmie = 0;
  for (int p = 0; p < nparts; ++p) {
    PartHost &h = H[p];
    PartDev &d = pd[p];
    d.nlam = h.nlam;
    d.nmc = h.nmc;
    d.ns = h.ns;
    d.nf = h.nf;
    d.samp0 = (int)sstat.size();
    d.mie0 = (int)mneed.size();
    d.out0 = (int)row_part.size();
    d.mscale = h.mscale;
    for (int ilam = 0; ilam < h.nlam; ++ilam) {
      row_part.push_back(p);
      double wvno = 2.0 * DHS_PI / in[p].lam[ilam];
      for (int l = 0; l < h.nmc; ++l) {
        double e1 = h.e1[(size_t)l * h.nlam + ilam], e2 = h.e2[(size_t)l * h.nlam + ilam];
        for (int k = 0; k < h.ns; ++k) {
          double r1 = h.r1[k];
          int need = 0;
          for (int i = 0; i < h.nf; ++i) {
            double rad = h.rad[(size_t)k * h.nf + i];
            int8_t st = S_DHS;
            if (h.f[i] == 0.0 || r1 * wvno > 10000.0) st = S_MIE;
            if (h.frac[l] == 0.0) {
              st = S_MIE; /* skipped by the accumulation, never evaluated */
            } else if (st == S_MIE) {
              need = 1;
            }
            srcore.push_back(h.rcore[(size_t)k * h.nf + i]);
            srshell.push_back(rad);
            swvno.push_back(wvno);
            smre.push_back(e1);
            smim.push_back(e2);
            sstat.push_back(st);
            if (st == S_DHS) maxnmx1 = std::max(maxnmx1, dhs_nmx1(rad, wvno, e1, -e2));
          }
          double lm = in[p].lam[ilam];
          if (r1 / lm >= 5000.0) lm = r1 / 5000.0;
          mrad.push_back(r1);
          mlam.push_back(lm);
          me1.push_back(e1);
          me2.push_back(e2);
          mneed.push_back(need);
        }
      }
    }
  }
  const int nsamp = (int)sstat.size();
  const int nslot = (int)mneed.size();
  const int nrows = (int)row_part.size();
  if (maxnmx1 + 1 > DHS_LL) maxnmx1 = DHS_LL; /* larger samples return Err inside */
  /* Mie term counts of every slot (any slot can be needed after a DHS
   * failure) */
  for (int q = 0; q < nslot; ++q) {
    int nmax, nfi, nD;
    mie_counts(mrad[q], mlam[q], me1[q], me2[q], &nmax, &nfi, &nD);
    maxmie = std::max(maxmie, std::max(nfi, nD));
  }
  const int dcap = maxnmx1 + 2;
  const int mcap = maxmie + 2;
  if ((long long)mcap > 50000000LL)
    return mcg_fail(ctx, MCG_ERR_LIMIT, "compute_part: Mie term count %d beyond the 5e7 limit", maxmie);

  std::vector<void *> own;
  cudaError_t ce = cudaSuccess;
  auto fail_free = [&](const char *what) {
    for (void *q : own) cudaFree(q);
    return mcg_fail(ctx, MCG_ERR_NOMEM, "compute_part: cudaMalloc of %s failed: %s", what, cudaGetErrorString(ce));
  };
#define ALLOC(T, n, name)                          \
  dev_alloc<T>(own, (size_t)(n), ce);              \
  if (ce != cudaSuccess) return fail_free(name)
  double *d_rcore = ALLOC(double, nsamp, "rcore");
  double *d_rshell = ALLOC(double, nsamp, "rshell");
  double *d_wvno = ALLOC(double, nsamp, "wvno");
  double *d_mre = ALLOC(double, nsamp, "mre");
  double *d_mim = ALLOC(double, nsamp, "mim");
  int8_t *d_stat = ALLOC(int8_t, nsamp, "status");
  double *d_sF = ALLOC(double, (size_t)nsamp * 4 * NA, "sample F");
  double *d_scs = ALLOC(double, (size_t)nsamp * 2, "sample cs");
  double *d_mrad = ALLOC(double, nslot, "mie rad");
  double *d_mlam = ALLOC(double, nslot, "mie lam");
  double *d_me1 = ALLOC(double, nslot, "mie e1");
  double *d_me2 = ALLOC(double, nslot, "mie e2");
  int *d_mneed = ALLOC(int, nslot, "mie need");
  double *d_mF = ALLOC(double, (size_t)nslot * 4 * NA, "mie F");
  double *d_mcs = ALLOC(double, (size_t)nslot * 2, "mie cs");
  int8_t *d_mok = ALLOC(int8_t, nslot, "mie ok");
  double *d_mu = ALLOC(double, 90, "mu");
  double *d_sinw = ALLOC(double, NA, "sinw");
  unsigned long long *d_next = ALLOC(unsigned long long, 2, "counters");
  PartDev *d_parts = ALLOC(PartDev, nparts, "parts");
  int *d_rowpart = ALLOC(int, nrows, "row map");
  double *d_kabs = ALLOC(double, nrows, "kabs");
  double *d_ksca = ALLOC(double, nrows, "ksca");
  double *d_kext = ALLOC(double, nrows, "kext");
  double *d_Fout = ALLOC(double, (size_t)nrows * 6 * NA, "F out");
  double *d_rhoav = ALLOC(double, nparts, "rho_av");
  /* per-part small arrays */
  std::vector<double> pflat;
  std::vector<size_t> off_frac(nparts), off_rho(nparts), off_r1(nparts), off_nr(nparts), off_wf(nparts);
  for (int p = 0; p < nparts; ++p) {
    off_frac[p] = pflat.size(); pflat.insert(pflat.end(), H[p].frac.begin(), H[p].frac.begin() + H[p].nmc);
    off_rho[p] = pflat.size(); pflat.insert(pflat.end(), H[p].rho.begin(), H[p].rho.begin() + H[p].nmc);
    off_r1[p] = pflat.size(); pflat.insert(pflat.end(), H[p].r1.begin(), H[p].r1.end());
    off_nr[p] = pflat.size(); pflat.insert(pflat.end(), H[p].nr.begin(), H[p].nr.end());
    off_wf[p] = pflat.size(); pflat.insert(pflat.end(), H[p].wf.begin(), H[p].wf.begin() + H[p].nf);
  }
  double *d_pflat = ALLOC(double, pflat.size(), "part tables");
#undef ALLOC
  for (int p = 0; p < nparts; ++p) {
    pd[p].frac = d_pflat + off_frac[p];
    pd[p].rho = d_pflat + off_rho[p];
    pd[p].r1 = d_pflat + off_r1[p];
    pd[p].nr = d_pflat + off_nr[p];
    pd[p].wf = d_pflat + off_wf[p];
  }
  cudaStream_t st = ctx->stream;
#define H2D(dst, src, n) cudaMemcpyAsync(dst, src, (size_t)(n) * sizeof(*(src)), cudaMemcpyHostToDevice, st)
  H2D(d_rcore, srcore.data(), nsamp);
  H2D(d_rshell, srshell.data(), nsamp);
  H2D(d_wvno, swvno.data(), nsamp);
  H2D(d_mre, smre.data(), nsamp);
  H2D(d_mim, smim.data(), nsamp);
  H2D(d_stat, sstat.data(), nsamp);
  H2D(d_mrad, mrad.data(), nslot);
  H2D(d_mlam, mlam.data(), nslot);
  H2D(d_me1, me1.data(), nslot);
  H2D(d_me2, me2.data(), nslot);
  H2D(d_mneed, mneed.data(), nslot);
  H2D(d_mu, mu, 90);
  H2D(d_sinw, sinw, NA);
  H2D(d_parts, pd.data(), nparts);
  H2D(d_rowpart, row_part.data(), nrows);
  H2D(d_pflat, pflat.data(), pflat.size());
#undef H2D
  cudaMemsetAsync(d_next, 0, 2 * sizeof(unsigned long long), st);
  cudaMemsetAsync(d_mok, 0, nslot, st);

  /* launch shapes: 4 warps per block, a multiple of the SM count; the number
   * of warps is bounded by the scratch budget */
  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  const size_t budget = (size_t)1 << 31; /* 2 GiB of down-recurrence scratch */
  auto warps_for = [&](size_t per_warp, int work) {
    long long w = std::min<long long>((long long)sms * 32, (long long)work);
    long long wb = (long long)(budget / std::max<size_t>(per_warp, 1));
    w = std::max<long long>(1, std::min(w, wb));
    return (int)w;
  };
  /* whole blocks of 4 warps: scratch is sliced per launched warp */
  int nw_dhs = (warps_for((size_t)4 * dcap * sizeof(cx), nsamp) + 3) / 4 * 4;
  int nw_mie = (warps_for((size_t)8 * mcap * sizeof(double), nslot) + 3) / 4 * 4;
  size_t scratch_bytes = std::max((size_t)nw_dhs * 4 * dcap * sizeof(cx), (size_t)nw_mie * 8 * mcap * sizeof(double));
  if (ctx->part_scratch.bytes < scratch_bytes) {
    if (ctx->part_scratch.p) cudaFree(ctx->part_scratch.p);
    ctx->part_scratch.p = nullptr;
    ctx->part_scratch.bytes = 0;
    ce = cudaMalloc(&ctx->part_scratch.p, scratch_bytes);
    if (ce != cudaSuccess) return fail_free("recurrence scratch");
    ctx->part_scratch.bytes = scratch_bytes;
  }
  SampleDev sd{d_rcore, d_rshell, d_wvno, d_mre, d_mim, d_stat, d_sF, d_scs, d_mneed, nsamp};
  int blocks = (nw_dhs + 3) / 4;
  dhs_kernel<<<blocks, 128, 0, st>>>(sd, d_mu, (cx *)ctx->part_scratch.p, dcap, d_next);
  /* a failed DHS sample marks its (part, lam, l, k) slot for the Mie pass */
  {
    /* status is tiny: bring it back and mark on the host */
    std::vector<int8_t> stat(nsamp);
    cudaMemcpyAsync(stat.data(), d_stat, nsamp, cudaMemcpyDeviceToHost, st);
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      for (void *q : own) cudaFree(q);
      return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part: DHS kernel failed: %s", cudaGetErrorString(ce));
    }
    bool changed = false;
    for (int p = 0; p < nparts; ++p) {
      const PartHost &h = H[p];
      for (int ilam = 0; ilam < h.nlam; ++ilam)
        for (int l = 0; l < h.nmc; ++l)
          for (int k = 0; k < h.ns; ++k) {
            int slot = pd[p].mie0 + (ilam * h.nmc + l) * h.ns + k;
            for (int i = 0; i < h.nf; ++i) {
              int s = pd[p].samp0 + ((ilam * h.nmc + l) * h.ns + k) * h.nf + i;
              if (stat[s] == S_DHS_ERR && !mneed[slot]) {
                mneed[slot] = 1;
                changed = true;
              }
            }
          }
    }
    int64_t nd = 0, nfail = 0, nm = 0;
    for (int p = 0; p < nparts; ++p) {
      const PartHost &h = H[p];
      int64_t pdhs = 0, pfail = 0, pmie = 0;
      for (int s = pd[p].samp0; s < pd[p].samp0 + h.nlam * h.nmc * h.ns * h.nf; ++s) {
        if (stat[s] == S_DHS) pdhs++;
        if (stat[s] == S_DHS_ERR) { pdhs++; pfail++; }
      }
      for (int q = pd[p].mie0; q < pd[p].mie0 + h.nlam * h.nmc * h.ns; ++q) pmie += mneed[q];
      out[p].n_dhs = pdhs;
      out[p].n_dhs_fail = pfail;
      out[p].n_mie = pmie;
      nd += pdhs; nfail += pfail; nm += pmie;
    }
    if (changed) cudaMemcpyAsync(d_mneed, mneed.data(), (size_t)nslot * sizeof(int), cudaMemcpyHostToDevice, st);
  }
  MieDev md{d_mrad, d_mlam, d_me1, d_me2, d_mneed, d_mF, d_mcs, d_mok, nslot};
  blocks = (nw_mie + 3) / 4;
  mie_kernel<<<blocks, 128, 0, st>>>(md, (double *)ctx->part_scratch.p, mcap, d_next + 1);
  AccDev ad{d_parts, nparts, d_rowpart, d_stat, d_sF, d_scs, d_mF, d_mcs, d_sinw, tot2,
            d_kabs, d_ksca, d_kext, d_Fout, d_rhoav, nrows};
  accum_kernel<<<(nrows + 3) / 4, 128, 0, st>>>(ad);
  ce = cudaGetLastError();
  std::vector<double> kabs(nrows), ksca(nrows), kext(nrows), Fo((size_t)nrows * 6 * NA), rhoav(nparts);
  std::vector<int8_t> mok(nslot);
  cudaMemcpyAsync(kabs.data(), d_kabs, nrows * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ksca.data(), d_ksca, nrows * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(kext.data(), d_kext, nrows * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(Fo.data(), d_Fout, Fo.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(rhoav.data(), d_rhoav, nparts * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(mok.data(), d_mok, nslot, cudaMemcpyDeviceToHost, st);
  cudaError_t se = cudaStreamSynchronize(st);
  for (void *q : own) cudaFree(q);
  if (ce != cudaSuccess || se != cudaSuccess)
    return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part: kernels failed: %s",
                    cudaGetErrorString(ce != cudaSuccess ? ce : se));
  for (int q = 0; q < nslot; ++q)
    if (mneed[q] && !mok[q])
      return mcg_fail(ctx, MCG_ERR_LIMIT, "compute_part: homogeneous-sphere fallback did not fit (slot %d)", q);
  for (int p = 0; p < nparts; ++p) {
    const int r0 = pd[p].out0, n = H[p].nlam;
    memcpy(out[p].kabs, kabs.data() + r0, n * sizeof(double));
    memcpy(out[p].ksca, ksca.data() + r0, n * sizeof(double));
    memcpy(out[p].kext, kext.data() + r0, n * sizeof(double));
    memcpy(out[p].F, Fo.data() + (size_t)r0 * 6 * NA, (size_t)n * 6 * NA * sizeof(double));
    out[p].rho_av = rhoav[p];
    out[p].mscale = H[p].mscale;
    out[p].rscale = H[p].rscale;
  }
  return MCG_OK;
}

/* ------------------------------------------------------------------------
 * ComputePart without device allocation (mcg_compute_part_static).
 *
 * For callers that must not allocate device memory themselves or through
 * this library: every device buffer of the call (staged inputs, per-sample
 * Mueller rows, Mie slots, recurrence scratch, outputs before the copy back)
 * is carved out of one file-scope array of MCG_STATIC_ARENA_BYTES.  The
 * array exists once per device for as long as the library is loaded.
 *
 * Wavelength rows are independent in ComputePart (ComputePart.f:318-447), so
 * a bin is processed in chunks of rows that fit the array; the kernels and
 * their per-row order are those of mcg_part_batch_impl, so the tables are
 * bit-identical to mcg_compute_part.
 *
 * The array keeps whatever the previous call left in it.  The work counters
 * and the Mie success flags are cleared on the stream before each chunk;
 * everything else is written before it is read.  Two calls whose work
 * overlaps on the GPU (two contexts on one device used from two host
 * threads) share the array and race; the call synchronises its stream
 * before returning, so calls made one after the other never overlap.
 * ---------------------------------------------------------------------- */
static __device__ __align__(256) unsigned char mcg_static_arena[MCG_STATIC_ARENA_BYTES];

namespace {

constexpr size_t kArenaBytes = (size_t)MCG_STATIC_ARENA_BYTES;

/* Device address of the array on the current device.  In host code the
 * symbol mcg_static_arena only names a host-side shadow; the kernels need
 * the address the runtime reports for the device.  It is looked up on every
 * call (a cheap runtime query) rather than cached for the process: after a
 * cudaDeviceReset, or when the primary context is released and created
 * again, the module is loaded anew and the array may sit at another
 * address.  The first lookup on a device loads the module, which is why the
 * first call on a device belongs before any stream capture. */
cudaError_t arena_address(unsigned char **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, mcg_static_arena);
  if (e != cudaSuccess) return e;
  *out = (unsigned char *)p;
  return cudaSuccess;
}

/* bump allocator over the array, 256-byte aligned pieces */
struct Carve {
  unsigned char *base;
  size_t off = 0, cap = 0;
  template <typename T>
  T *take(size_t n) {
    size_t bytes = (std::max<size_t>(n, 1) * sizeof(T) + 255) & ~(size_t)255;
    T *p = (T *)(base + off);
    off += bytes;
    return p;
  }
};

inline size_t padded(size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) & ~(size_t)255; }

}  // namespace

mcg_status mcg_part_static_impl(mcg_ctx *ctx, const mcg_part_in *in, mcg_part_out *out) {
  if (!in || !out) return mcg_fail(ctx, MCG_ERR_ARG, "compute_part_static: non-null in/out required");
  PartHost h;
  {
    std::string why;
    if (!part_setup(*in, h, why)) return mcg_fail(ctx, MCG_ERR_ARG, "%s", why.c_str());
  }
  if (!out->kabs || !out->ksca || !out->kext || !out->F)
    return mcg_fail(ctx, MCG_ERR_ARG, "compute_part_static: null output array");
  const int nlam = h.nlam, nmc = h.nmc, ns = h.ns, nf = h.nf;
  const long long per_row_samp = (long long)nmc * ns * nf, per_row_slot = (long long)nmc * ns;

  double mu[90], sinw[NA], tot2 = 0.0;
  for (int i = 1; i <= 90; ++i) mu[i - 1] = cos(((double)i - 0.5) / (double)(NA / 2) * DHS_PI / 2.0);
  for (int j = 1; j <= NA; ++j) sinw[j - 1] = sin(DHS_PI * ((double)j - 0.5) / (double)NA);
  for (int j = 0; j < NA; ++j) tot2 = tot2 + sinw[j];

  /* recurrence lengths over the whole bin (as mcg_part_batch_impl) */
  int maxnmx1 = 150, maxmie = 0;
  for (int ilam = 0; ilam < nlam; ++ilam) {
    const double wvno = 2.0 * DHS_PI / in->lam[ilam];
    for (int l = 0; l < nmc; ++l) {
      const double e1 = h.e1[(size_t)l * nlam + ilam], e2 = h.e2[(size_t)l * nlam + ilam];
      for (int k = 0; k < ns; ++k) {
        const double r1 = h.r1[k];
        for (int i = 0; i < nf; ++i) {
          const bool mie = h.f[i] == 0.0 || r1 * wvno > 10000.0 || h.frac[l] == 0.0;
          if (!mie) maxnmx1 = std::max(maxnmx1, dhs_nmx1(h.rad[(size_t)k * nf + i], wvno, e1, -e2));
        }
        double lm = in->lam[ilam];
        if (r1 / lm >= 5000.0) lm = r1 / 5000.0;
        int nmax, nfi, nD;
        mie_counts(r1, lm, e1, e2, &nmax, &nfi, &nD);
        maxmie = std::max(maxmie, std::max(nfi, nD));
      }
    }
  }
  if (maxnmx1 + 1 > DHS_LL) maxnmx1 = DHS_LL;
  const int dcap = maxnmx1 + 2, mcap = maxmie + 2;
  if ((long long)mcap > 50000000LL)
    return mcg_fail(ctx, MCG_ERR_LIMIT, "compute_part_static: Mie term count %d beyond the 5e7 limit", maxmie);
  const size_t per_warp = std::max((size_t)4 * dcap * sizeof(cx), (size_t)8 * mcap * sizeof(double));

  /* bytes: fixed part, per wavelength row, per warp of recurrence scratch */
  std::vector<double> pflat;
  pflat.insert(pflat.end(), h.frac.begin(), h.frac.begin() + nmc);
  pflat.insert(pflat.end(), h.rho.begin(), h.rho.begin() + nmc);
  pflat.insert(pflat.end(), h.r1.begin(), h.r1.end());
  pflat.insert(pflat.end(), h.nr.begin(), h.nr.end());
  pflat.insert(pflat.end(), h.wf.begin(), h.wf.begin() + nf);
  const size_t fixed = padded(90 * 8) + padded(NA * 8) + padded(16) + padded(sizeof(PartDev)) +
                       padded(pflat.size() * 8) + padded(8) /* rho_av */;
  /* 5 staged doubles, status, 4x180 Mueller, 2 cross sections per sample;
   * 4 staged doubles, need flag, 4x180 Mueller, 2 cross sections, ok flag
   * per Mie slot; row map, 3 opacities, 6x180 Mueller per row; each of the
   * 21 row-sized arrays may lose up to 255 bytes to alignment */
  const size_t per_row = (size_t)per_row_samp * (5 * 8 + 1 + 4 * NA * 8 + 2 * 8) +
                         (size_t)per_row_slot * (4 * 8 + 4 + 4 * NA * 8 + 2 * 8 + 1) + 4 + 3 * 8 + 6 * NA * 8;
  const size_t align_slack = 21 * 256;
  if (fixed + align_slack + per_row + 4 * per_warp > kArenaBytes)
    return mcg_fail(ctx, MCG_ERR_LIMIT,
                    "compute_part_static: one wavelength row needs %zu bytes of device working memory "
                    "(%lld samples, %zu bytes of recurrence scratch for 4 warps); the static array holds %zu",
                    fixed + align_slack + per_row + 4 * per_warp, per_row_samp, 4 * per_warp, kArenaBytes);
  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  /* scratch for up to one warp per sample of a chunk, at most 32 warps per
   * SM, at most half the array; the rest holds rows */
  size_t want_warps = std::min<size_t>((size_t)sms * 32, (size_t)std::max<long long>(4, per_row_samp * nlam));
  size_t scratch = std::min(want_warps * per_warp, kArenaBytes / 2);
  scratch = std::max(scratch, 4 * per_warp);
  size_t rows_fit = (kArenaBytes - fixed - align_slack - scratch) / per_row;
  if (rows_fit < 1) {
    scratch = 4 * per_warp;
    rows_fit = (kArenaBytes - fixed - align_slack - scratch) / per_row;
  }
  const int nlc_max = (int)std::min<size_t>(rows_fit, (size_t)nlam);
  const size_t rows_bytes = (size_t)nlc_max * per_row + align_slack;
  int nw = (int)(std::min((kArenaBytes - fixed - rows_bytes) / per_warp, (size_t)sms * 32) / 4 * 4);
  if (nw < 4) nw = 4;

  unsigned char *arena = nullptr;
  cudaError_t ce = arena_address(&arena);
  if (ce != cudaSuccess)
    return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part_static: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(ce));
  cudaStream_t st = ctx->stream;
  Carve cv{arena, 0, kArenaBytes};
  double *d_mu = cv.take<double>(90);
  double *d_sinw = cv.take<double>(NA);
  unsigned long long *d_next = cv.take<unsigned long long>(2);
  PartDev *d_part = cv.take<PartDev>(1);
  double *d_pflat = cv.take<double>(pflat.size());
  double *d_rhoav = cv.take<double>(1);
  const size_t chunk_base = cv.off;

  cudaMemcpyAsync(d_mu, mu, sizeof mu, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_sinw, sinw, sizeof sinw, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_pflat, pflat.data(), pflat.size() * sizeof(double), cudaMemcpyHostToDevice, st);

  int64_t n_dhs = 0, n_fail = 0, n_mie = 0;
  std::vector<double> srcore, srshell, swvno, smre, smim, mrad, mlam, me1, me2;
  std::vector<int8_t> sstat, stat, mok;
  std::vector<int> mneed, rowpart;
  for (int c0 = 0; c0 < nlam; c0 += nlc_max) {
    const int nlc = std::min(nlc_max, nlam - c0);
    srcore.clear(); srshell.clear(); swvno.clear(); smre.clear(); smim.clear(); sstat.clear();
    mrad.clear(); mlam.clear(); me1.clear(); me2.clear(); mneed.clear();
    for (int ilam = c0; ilam < c0 + nlc; ++ilam) {
      const double wvno = 2.0 * DHS_PI / in->lam[ilam];
      for (int l = 0; l < nmc; ++l) {
        const double e1 = h.e1[(size_t)l * nlam + ilam], e2 = h.e2[(size_t)l * nlam + ilam];
        for (int k = 0; k < ns; ++k) {
          const double r1 = h.r1[k];
          int need = 0;
          for (int i = 0; i < nf; ++i) {
            int8_t s8 = S_DHS;
            if (h.f[i] == 0.0 || r1 * wvno > 10000.0) s8 = S_MIE;
            if (h.frac[l] == 0.0) {
              s8 = S_MIE;
            } else if (s8 == S_MIE) {
              need = 1;
            }
            srcore.push_back(h.rcore[(size_t)k * nf + i]);
            srshell.push_back(h.rad[(size_t)k * nf + i]);
            swvno.push_back(wvno);
            smre.push_back(e1);
            smim.push_back(e2);
            sstat.push_back(s8);
          }
          double lm = in->lam[ilam];
          if (r1 / lm >= 5000.0) lm = r1 / 5000.0;
          mrad.push_back(r1);
          mlam.push_back(lm);
          me1.push_back(e1);
          me2.push_back(e2);
          mneed.push_back(need);
        }
      }
    }
    const int nsamp = (int)sstat.size(), nslot = (int)mneed.size();
    cv.off = chunk_base;
    double *d_rcore = cv.take<double>(nsamp), *d_rshell = cv.take<double>(nsamp);
    double *d_wvno = cv.take<double>(nsamp), *d_mre = cv.take<double>(nsamp), *d_mim = cv.take<double>(nsamp);
    int8_t *d_stat = cv.take<int8_t>(nsamp);
    double *d_sF = cv.take<double>((size_t)nsamp * 4 * NA), *d_scs = cv.take<double>((size_t)nsamp * 2);
    double *d_mrad = cv.take<double>(nslot), *d_mlam = cv.take<double>(nslot);
    double *d_me1 = cv.take<double>(nslot), *d_me2 = cv.take<double>(nslot);
    int *d_mneed = cv.take<int>(nslot);
    double *d_mF = cv.take<double>((size_t)nslot * 4 * NA), *d_mcs = cv.take<double>((size_t)nslot * 2);
    int8_t *d_mok = cv.take<int8_t>(nslot);
    int *d_rowpart = cv.take<int>(nlc);
    double *d_kabs = cv.take<double>(nlc), *d_ksca = cv.take<double>(nlc), *d_kext = cv.take<double>(nlc);
    double *d_Fout = cv.take<double>((size_t)nlc * 6 * NA);
    const size_t scratch_off = cv.off;
    if (scratch_off + (size_t)nw * per_warp > kArenaBytes)
      return mcg_fail(ctx, MCG_ERR_LIMIT, "compute_part_static: internal layout exceeds the static array");

    /* the chunk's rows are local (0..nlc-1); offsets shift the absolute
     * wavelength index ilam = row + c0 onto them */
    PartDev pd;
    pd.nlam = nlam;
    pd.nmc = nmc;
    pd.ns = ns;
    pd.nf = nf;
    pd.samp0 = -(int)(c0 * per_row_samp);
    pd.mie0 = -(int)(c0 * per_row_slot);
    pd.out0 = -c0;
    pd.mscale = h.mscale;
    pd.frac = d_pflat;
    pd.rho = d_pflat + nmc;
    pd.r1 = d_pflat + 2 * nmc;
    pd.nr = d_pflat + 2 * nmc + ns;
    pd.wf = d_pflat + 2 * nmc + ns + (size_t)nmc * ns;
    rowpart.assign(nlc, 0);
#define H2D(dst, src, n) cudaMemcpyAsync(dst, src, (size_t)(n) * sizeof(*(src)), cudaMemcpyHostToDevice, st)
    H2D(d_rcore, srcore.data(), nsamp);
    H2D(d_rshell, srshell.data(), nsamp);
    H2D(d_wvno, swvno.data(), nsamp);
    H2D(d_mre, smre.data(), nsamp);
    H2D(d_mim, smim.data(), nsamp);
    H2D(d_stat, sstat.data(), nsamp);
    H2D(d_mrad, mrad.data(), nslot);
    H2D(d_mlam, mlam.data(), nslot);
    H2D(d_me1, me1.data(), nslot);
    H2D(d_me2, me2.data(), nslot);
    H2D(d_mneed, mneed.data(), nslot);
    H2D(d_part, &pd, 1);
    H2D(d_rowpart, rowpart.data(), nlc);
#undef H2D
    /* what the previous call or chunk left behind must not count */
    cudaMemsetAsync(d_next, 0, 2 * sizeof(unsigned long long), st);
    cudaMemsetAsync(d_mok, 0, nslot, st);

    SampleDev sd{d_rcore, d_rshell, d_wvno, d_mre, d_mim, d_stat, d_sF, d_scs, d_mneed, nsamp};
    const int nw_dhs = std::min(nw, (nsamp + 3) / 4 * 4);
    dhs_kernel<<<(nw_dhs + 3) / 4, 128, 0, st>>>(sd, d_mu, (cx *)(arena + scratch_off), dcap, d_next);
    stat.resize(nsamp);
    cudaMemcpyAsync(stat.data(), d_stat, nsamp, cudaMemcpyDeviceToHost, st);
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess)
      return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part_static: DHS kernel failed: %s", cudaGetErrorString(ce));
    bool changed = false;
    for (int q = 0; q < nslot; ++q)
      for (int i = 0; i < nf; ++i) {
        const int8_t s8 = stat[(size_t)q * nf + i];
        if (s8 == S_DHS) n_dhs++;
        if (s8 == S_DHS_ERR) {
          n_dhs++;
          n_fail++;
          if (!mneed[q]) {
            mneed[q] = 1;
            changed = true;
          }
        }
      }
    for (int q = 0; q < nslot; ++q) n_mie += mneed[q];
    if (changed) cudaMemcpyAsync(d_mneed, mneed.data(), (size_t)nslot * sizeof(int), cudaMemcpyHostToDevice, st);
    MieDev md{d_mrad, d_mlam, d_me1, d_me2, d_mneed, d_mF, d_mcs, d_mok, nslot};
    const int nw_mie = std::min(nw, (nslot + 3) / 4 * 4);
    mie_kernel<<<(nw_mie + 3) / 4, 128, 0, st>>>(md, (double *)(arena + scratch_off), mcap, d_next + 1);
    AccDev ad{d_part, 1, d_rowpart, d_stat, d_sF, d_scs, d_mF, d_mcs, d_sinw, tot2,
              d_kabs, d_ksca, d_kext, d_Fout, d_rhoav, nlc};
    accum_kernel<<<(nlc + 3) / 4, 128, 0, st>>>(ad);
    ce = cudaGetLastError();
    if (ce != cudaSuccess)
      return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part_static: launch failed: %s", cudaGetErrorString(ce));
    mok.resize(nslot);
    cudaMemcpyAsync(out->kabs + c0, d_kabs, nlc * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out->ksca + c0, d_ksca, nlc * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out->kext + c0, d_kext, nlc * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out->F + (size_t)c0 * 6 * NA, d_Fout, (size_t)nlc * 6 * NA * sizeof(double),
                    cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(mok.data(), d_mok, nslot, cudaMemcpyDeviceToHost, st);
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess)
      return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part_static: kernels failed: %s", cudaGetErrorString(ce));
    for (int q = 0; q < nslot; ++q)
      if (mneed[q] && !mok[q])
        return mcg_fail(ctx, MCG_ERR_LIMIT, "compute_part_static: homogeneous-sphere fallback did not fit (slot %d)",
                        q + (int)(c0 * per_row_slot));
  }
  double rho_av = 0.0;
  cudaMemcpyAsync(&rho_av, d_rhoav, sizeof(double), cudaMemcpyDeviceToHost, st);
  ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess)
    return mcg_fail(ctx, MCG_ERR_CUDA, "compute_part_static: copy failed: %s", cudaGetErrorString(ce));
  out->rho_av = rho_av;
  out->mscale = h.mscale;
  out->rscale = h.rscale;
  out->n_dhs = n_dhs;
  out->n_dhs_fail = n_fail;
  out->n_mie = n_mie;
  return MCG_OK;
}

/* ------------------------------------------------------------------------
 * Training targets of the opacity surrogate (mcg_surrogate_targets).
 *
 * Each sample is one ComputePart call for a single grain size: one .lnk
 * material (n, k at one wavelength) Bruggeman-blended with a vacuum
 * fraction `porosity` (ComputePart.f:227-252), ns = 1, nf DHS filling
 * fractions on [0.01, fmax] (ComputePart.f:266-274), no abundance
 * normalisation.  The samples go through the same dhs_kernel, mie_kernel
 * and accum_kernel as mcg_compute_part (one output row per sample), and
 * moments_kernel reduces each row's Mueller elements to the targets:
 *   [0] log10 kappa_abs, [1] log10 kappa_sca (cm^2/g),
 *   [2 + l - 1] chi_l, l = 1..12  moments of F11: sum_j F11_j P_l(mu_j) w_j
 *   [14 + l]    beta_l, l = 0..12 moments of F12,
 *   [27 + l]    gamma_l, l = 0..12 moments of F33,
 *   [40 + l]    delta_l, l = 0..12 moments of F34, all / sum_j F11_j w_j,
 *   mu_j = cos((j + 1/2) deg), w_j = sin((j + 1/2) deg); [53..63] = 0.
 * (F22 = F11 and F44 = F33 for the spheres of DHS and Mie.)
 * ---------------------------------------------------------------------- */
namespace {

constexpr int SURR_L = 12;
constexpr int SURR_OUT = 64; /* targets per sample */

__global__ void __launch_bounds__(128) moments_kernel(int nrows, const double *kabs, const double *ksca,
                                                      const double *Fout, float *out) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= nrows) return;
  double s11[SURR_L + 1], s12[SURR_L + 1], s33[SURR_L + 1], s34[SURR_L + 1];
#pragma unroll
  for (int l = 0; l <= SURR_L; ++l) s11[l] = s12[l] = s33[l] = s34[l] = 0.0;
  for (int j = lane; j < NA; j += WARP) {
    const double th = DHS_PI * ((double)j + 0.5) / (double)NA;
    const double mu = cos(th), w = sin(th);
    const double f11 = Fout[((size_t)row * 6 + 0) * NA + j] * w;
    const double f12 = Fout[((size_t)row * 6 + 1) * NA + j] * w;
    const double f33 = Fout[((size_t)row * 6 + 3) * NA + j] * w;
    const double f34 = Fout[((size_t)row * 6 + 4) * NA + j] * w;
    double p0 = 1.0, p1 = mu;
    s11[0] += f11;
    s12[0] += f12;
    s33[0] += f33;
    s34[0] += f34;
    s11[1] += f11 * p1;
    s12[1] += f12 * p1;
    s33[1] += f33 * p1;
    s34[1] += f34 * p1;
#pragma unroll
    for (int l = 1; l < SURR_L; ++l) {
      const double p2 = ((2.0 * l + 1.0) * mu * p1 - (double)l * p0) / (double)(l + 1);
      s11[l + 1] += f11 * p2;
      s12[l + 1] += f12 * p2;
      s33[l + 1] += f33 * p2;
      s34[l + 1] += f34 * p2;
      p0 = p1;
      p1 = p2;
    }
  }
#pragma unroll
  for (int l = 0; l <= SURR_L; ++l)
    for (int s = 16; s > 0; s >>= 1) {
      s11[l] += __shfl_down_sync(0xffffffffu, s11[l], s);
      s12[l] += __shfl_down_sync(0xffffffffu, s12[l], s);
      s33[l] += __shfl_down_sync(0xffffffffu, s33[l], s);
      s34[l] += __shfl_down_sync(0xffffffffu, s34[l], s);
    }
  if (lane == 0) {
    float *o = out + (size_t)row * SURR_OUT;
    o[0] = (float)log10(fmax(kabs[row], 1e-30));
    o[1] = (float)log10(fmax(ksca[row], 1e-30));
    const double inv = s11[0] > 0.0 ? 1.0 / s11[0] : 0.0;
    for (int l = 1; l <= SURR_L; ++l) o[1 + l] = (float)(s11[l] * inv);
    for (int l = 0; l <= SURR_L; ++l) o[14 + l] = (float)(s12[l] * inv);
    for (int l = 0; l <= SURR_L; ++l) o[27 + l] = (float)(s33[l] * inv);
    for (int l = 0; l <= SURR_L; ++l) o[40 + l] = (float)(s34[l] * inv);
    for (int k = 53; k < SURR_OUT; ++k) o[k] = 0.0f;
  }
}

}  // namespace

mcg_status mcg_surrogate_targets_impl(mcg_ctx *ctx, int64_t n, const double *in6, double rho, int nf, float *out) {
  if (n < 1 || !in6 || !out || nf < 1 || nf > 64 || !(rho > 0.0))
    return mcg_fail(ctx, MCG_ERR_ARG, "surrogate_targets: n >= 1, 1 <= nf <= 64, rho > 0 and non-null arrays");
  for (int64_t s = 0; s < n; ++s) {
    const double *q = in6 + 6 * s;
    if (!(q[0] > 0.0) || !(q[1] > 0.0) || !(q[2] > 0.0) || !(q[3] >= 0.0) || !(q[4] >= 0.0) || !(q[4] < 1.0) ||
        !(q[5] >= 0.0) || !(q[5] < 1.0))
      return mcg_fail(ctx, MCG_ERR_ARG, "surrogate_targets: sample %lld outside the physical range", (long long)s);
  }
  /* order by size parameter so each chunk's recurrence lengths are alike */
  std::vector<int64_t> order((size_t)n);
  for (int64_t s = 0; s < n; ++s) order[(size_t)s] = s;
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return in6[6 * a] / in6[6 * a + 1] < in6[6 * b] / in6[6 * b + 1];
  });
  double mu[90], sinw[NA], tot2 = 0.0;
  for (int i = 1; i <= 90; ++i) mu[i - 1] = cos(((double)i - 0.5) / (double)(NA / 2) * DHS_PI / 2.0);
  for (int j = 1; j <= NA; ++j) sinw[j - 1] = sin(DHS_PI * ((double)j - 0.5) / (double)NA);
  for (int j = 0; j < NA; ++j) tot2 = tot2 + sinw[j];
  const int64_t CH = 65536;
  cudaStream_t st = ctx->stream;
  const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
  std::vector<float> tout;
  for (int64_t c0 = 0; c0 < n; c0 += CH) {
    const int m = (int)std::min<int64_t>(CH, n - c0);
    std::vector<double> srcore, srshell, swvno, smre, smim, mrad, mlam, me1, me2, pflat;
    std::vector<int8_t> sstat;
    std::vector<int> mneed, rowpart(m);
    std::vector<PartDev> pd(m);
    std::vector<size_t> poff(m);
    int maxnmx1 = 150, maxmie = 0;
    for (int r = 0; r < m; ++r) {
      const double *q = in6 + 6 * order[(size_t)(c0 + r)];
      const double a = q[0], lam = q[1], por = q[4], fmx = q[5];
      /* Bruggeman blend with vacuum (ComputePart.f:227-252), nm = 1 */
      double e1b, e2b;
      {
        const double e1s[2] = {q[2], 1.0}, e2s[2] = {q[3], 0.0}, ab[2] = {1.0 - por, por};
        blender(e1s, e2s, ab, 2, &e1b, &e2b);
      }
      const double rav = (1.0 - por) * rho;
      /* filling fractions (ComputePart.f:266-274) */
      int nfs = nf;
      std::vector<double> f(nf, 0.0), wf(nf, 0.0);
      if (fmx == 0.0) nfs = 1;
      if (nfs > 1 && fmx > 0.01) {
        gauleg2(0.01, fmx, f.data(), wf.data(), nfs);
      } else if (fmx == 0.0) {
        f[0] = 0.0;
        wf[0] = 1.0;
      } else {
        nfs = 1;
        f[0] = fmx;
        wf[0] = 1.0;
      }
      const double wvno = 2.0 * DHS_PI / lam;
      PartDev &d = pd[r];
      d.nlam = 1;
      d.nmc = 1;
      d.ns = 1;
      d.nf = nfs;
      d.samp0 = (int)sstat.size();
      d.mie0 = (int)mneed.size();
      d.out0 = r;
      d.mscale = 1.0;
      poff[r] = pflat.size();
      pflat.push_back(1.0); /* frac */
      pflat.push_back(rav); /* rho */
      pflat.push_back(a);   /* r1 */
      pflat.push_back(1.0); /* nr */
      for (int i = 0; i < nfs; ++i) pflat.push_back(wf[i]);
      rowpart[r] = r;
      int need = 0;
      for (int i = 0; i < nfs; ++i) {
        const double rad = a / pow(1.0 - f[i], 1.0 / 3.0);
        int8_t s8 = S_DHS;
        if (f[i] == 0.0 || a * wvno > 10000.0) {
          s8 = S_MIE;
          need = 1;
        }
        srcore.push_back(f[i] > 0.0 ? rad * pow(f[i], 1.0 / 3.0) : 0.0);
        srshell.push_back(rad);
        swvno.push_back(wvno);
        smre.push_back(e1b);
        smim.push_back(e2b);
        sstat.push_back(s8);
        if (s8 == S_DHS) maxnmx1 = std::max(maxnmx1, dhs_nmx1(rad, wvno, e1b, -e2b));
      }
      double lm = lam;
      if (a / lm >= 5000.0) lm = a / 5000.0;
      mrad.push_back(a);
      mlam.push_back(lm);
      me1.push_back(e1b);
      me2.push_back(e2b);
      mneed.push_back(need);
      int nmax, nfi, nD;
      mie_counts(a, lm, e1b, e2b, &nmax, &nfi, &nD);
      maxmie = std::max(maxmie, std::max(nfi, nD));
    }
    const int nsamp = (int)sstat.size(), nslot = (int)mneed.size();
    if (maxnmx1 + 1 > DHS_LL) maxnmx1 = DHS_LL;
    const int dcap = maxnmx1 + 2, mcap = maxmie + 2;
    if ((long long)mcap > 50000000LL)
      return mcg_fail(ctx, MCG_ERR_LIMIT, "surrogate_targets: Mie term count %d beyond the 5e7 limit", maxmie);
    std::vector<void *> own;
    cudaError_t ce = cudaSuccess;
    auto fail_free = [&](const char *what) {
      for (void *p : own) cudaFree(p);
      return mcg_fail(ctx, MCG_ERR_NOMEM, "surrogate_targets: cudaMalloc of %s failed: %s", what,
                      cudaGetErrorString(ce));
    };
#define ALLOC(T, cnt, name)               \
  dev_alloc<T>(own, (size_t)(cnt), ce);   \
  if (ce != cudaSuccess) return fail_free(name)
    double *d_rcore = ALLOC(double, nsamp, "rcore");
    double *d_rshell = ALLOC(double, nsamp, "rshell");
    double *d_wvno = ALLOC(double, nsamp, "wvno");
    double *d_mre = ALLOC(double, nsamp, "mre");
    double *d_mim = ALLOC(double, nsamp, "mim");
    int8_t *d_stat = ALLOC(int8_t, nsamp, "status");
    double *d_sF = ALLOC(double, (size_t)nsamp * 4 * NA, "sample F");
    double *d_scs = ALLOC(double, (size_t)nsamp * 2, "sample cs");
    double *d_mrad = ALLOC(double, nslot, "mie rad");
    double *d_mlam = ALLOC(double, nslot, "mie lam");
    double *d_me1 = ALLOC(double, nslot, "mie e1");
    double *d_me2 = ALLOC(double, nslot, "mie e2");
    int *d_mneed = ALLOC(int, nslot, "mie need");
    double *d_mF = ALLOC(double, (size_t)nslot * 4 * NA, "mie F");
    double *d_mcs = ALLOC(double, (size_t)nslot * 2, "mie cs");
    int8_t *d_mok = ALLOC(int8_t, nslot, "mie ok");
    double *d_mu = ALLOC(double, 90, "mu");
    double *d_sinw = ALLOC(double, NA, "sinw");
    unsigned long long *d_next = ALLOC(unsigned long long, 2, "counters");
    PartDev *d_parts = ALLOC(PartDev, m, "parts");
    int *d_rowpart = ALLOC(int, m, "row map");
    double *d_kabs = ALLOC(double, m, "kabs");
    double *d_ksca = ALLOC(double, m, "ksca");
    double *d_kext = ALLOC(double, m, "kext");
    double *d_Fout = ALLOC(double, (size_t)m * 6 * NA, "F out");
    double *d_rhoav = ALLOC(double, m, "rho_av");
    double *d_pflat = ALLOC(double, pflat.size(), "part tables");
    float *d_out = ALLOC(float, (size_t)m * SURR_OUT, "targets");
#undef ALLOC
    for (int r = 0; r < m; ++r) {
      double *b = d_pflat + poff[r];
      pd[r].frac = b;
      pd[r].rho = b + 1;
      pd[r].r1 = b + 2;
      pd[r].nr = b + 3;
      pd[r].wf = b + 4;
    }
#define H2D(dst, src, cnt) cudaMemcpyAsync(dst, src, (size_t)(cnt) * sizeof(*(src)), cudaMemcpyHostToDevice, st)
    H2D(d_rcore, srcore.data(), nsamp);
    H2D(d_rshell, srshell.data(), nsamp);
    H2D(d_wvno, swvno.data(), nsamp);
    H2D(d_mre, smre.data(), nsamp);
    H2D(d_mim, smim.data(), nsamp);
    H2D(d_stat, sstat.data(), nsamp);
    H2D(d_mrad, mrad.data(), nslot);
    H2D(d_mlam, mlam.data(), nslot);
    H2D(d_me1, me1.data(), nslot);
    H2D(d_me2, me2.data(), nslot);
    H2D(d_mneed, mneed.data(), nslot);
    H2D(d_mu, mu, 90);
    H2D(d_sinw, sinw, NA);
    H2D(d_parts, pd.data(), m);
    H2D(d_rowpart, rowpart.data(), m);
    H2D(d_pflat, pflat.data(), pflat.size());
#undef H2D
    cudaMemsetAsync(d_next, 0, 2 * sizeof(unsigned long long), st);
    cudaMemsetAsync(d_mok, 0, nslot, st);
    const size_t budget = (size_t)1 << 31;
    auto warps_for = [&](size_t per_warp, int work) {
      long long w = std::min<long long>((long long)sms * 32, (long long)work);
      long long wb = (long long)(budget / std::max<size_t>(per_warp, 1));
      return (int)std::max<long long>(1, std::min(w, wb));
    };
    const int nw_dhs = (warps_for((size_t)4 * dcap * sizeof(cx), nsamp) + 3) / 4 * 4;
    const int nw_mie = (warps_for((size_t)8 * mcap * sizeof(double), nslot) + 3) / 4 * 4;
    const size_t scratch_bytes =
        std::max((size_t)nw_dhs * 4 * dcap * sizeof(cx), (size_t)nw_mie * 8 * mcap * sizeof(double));
    if (ctx->part_scratch.bytes < scratch_bytes) {
      if (ctx->part_scratch.p) cudaFree(ctx->part_scratch.p);
      ctx->part_scratch.p = nullptr;
      ctx->part_scratch.bytes = 0;
      ce = cudaMalloc(&ctx->part_scratch.p, scratch_bytes);
      if (ce != cudaSuccess) return fail_free("recurrence scratch");
      ctx->part_scratch.bytes = scratch_bytes;
    }
    SampleDev sd{d_rcore, d_rshell, d_wvno, d_mre, d_mim, d_stat, d_sF, d_scs, d_mneed, nsamp};
    dhs_kernel<<<(nw_dhs + 3) / 4, 128, 0, st>>>(sd, d_mu, (cx *)ctx->part_scratch.p, dcap, d_next);
    std::vector<int8_t> stat(nsamp);
    cudaMemcpyAsync(stat.data(), d_stat, nsamp, cudaMemcpyDeviceToHost, st);
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      for (void *p : own) cudaFree(p);
      return mcg_fail(ctx, MCG_ERR_CUDA, "surrogate_targets: DHS kernel failed: %s", cudaGetErrorString(ce));
    }
    bool changed = false;
    for (int r = 0; r < m; ++r)
      for (int i = 0; i < pd[r].nf; ++i)
        if (stat[pd[r].samp0 + i] == S_DHS_ERR && !mneed[r]) {
          mneed[r] = 1;
          changed = true;
        }
    if (changed) cudaMemcpyAsync(d_mneed, mneed.data(), (size_t)nslot * sizeof(int), cudaMemcpyHostToDevice, st);
    MieDev md{d_mrad, d_mlam, d_me1, d_me2, d_mneed, d_mF, d_mcs, d_mok, nslot};
    mie_kernel<<<(nw_mie + 3) / 4, 128, 0, st>>>(md, (double *)ctx->part_scratch.p, mcap, d_next + 1);
    AccDev ad{d_parts, m, d_rowpart, d_stat, d_sF, d_scs, d_mF, d_mcs, d_sinw, tot2,
              d_kabs, d_ksca, d_kext, d_Fout, d_rhoav, m};
    accum_kernel<<<(m + 3) / 4, 128, 0, st>>>(ad);
    moments_kernel<<<(m + 3) / 4, 128, 0, st>>>(m, d_kabs, d_ksca, d_Fout, d_out);
    ce = cudaGetLastError();
    tout.resize((size_t)m * SURR_OUT);
    std::vector<int8_t> mok(nslot);
    cudaMemcpyAsync(tout.data(), d_out, tout.size() * sizeof(float), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(mok.data(), d_mok, nslot, cudaMemcpyDeviceToHost, st);
    cudaError_t se = cudaStreamSynchronize(st);
    for (void *p : own) cudaFree(p);
    if (ce != cudaSuccess || se != cudaSuccess)
      return mcg_fail(ctx, MCG_ERR_CUDA, "surrogate_targets: kernels failed: %s",
                      cudaGetErrorString(ce != cudaSuccess ? ce : se));
    for (int q = 0; q < nslot; ++q)
      if (mneed[q] && !mok[q])
        return mcg_fail(ctx, MCG_ERR_LIMIT, "surrogate_targets: homogeneous-sphere fallback did not fit");
    for (int r = 0; r < m; ++r)
      memcpy(out + (size_t)SURR_OUT * order[(size_t)(c0 + r)], tout.data() + (size_t)r * SURR_OUT,
             SURR_OUT * sizeof(float));
  }
  return MCG_OK;
}
