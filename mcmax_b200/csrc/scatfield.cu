/*
 * scatfield.cu -- the scattered-light field of the ray tracer (TraceMono,
 * TraceMono.f:583-914), one field per wavelength and inclination.
 *
 *   sf_opac_kernel     one thread per cell: Kabs, Kext, Ksca, albedo at the
 *                      wavelength and EmissionDistribution's thermal weight
 *   sf_mueller_kernel  one thread per (cell, element): the cell's mixed
 *                      Mueller matrix (full-Mueller fields)
 *   sf_exit_kernel     one thread per cell: the exit depth over nexits
 *                      directions and the visibility weight exp(-tauexit)
 *   (host)             the running sum of the weighted emission in the
 *                      reference's cell order, for emitposition's choice
 *   sf_star_kernel     one warp per starlight packet (MakeStarScatter,
 *                      TraceMono.f:1585-1770): the single-scattered field of
 *                      the direct starlight along a straight path
 *   sf_mc_kernel       one warp per packet (emitposition, trace2dmono,
 *                      makescattfield, the albedo roulette and scatangle;
 *                      TraceMono.f:792-880, 1124-1560)
 *
 * In the packet kernels all 32 lanes follow the packet (they draw the same
 * Philox stream, so they agree on every step) and split the work that the
 * reference does per observer direction: the 180 scattering-angle indices
 * and Stokes rotations of a flight, and the 180 deposits of a path segment
 * into the folded azimuth bins, which lanes add with atomics.
 *
 * Packet p of a field draws the stream (key, p): starlight packets
 * p = 0..nstar-1, Monte Carlo packets nstar + 0..nphot-1; the key is the
 * call's seed plus the number of fields computed before in the call.
 * Where the reference evaluates Albedo**0.25 with pow, this takes the
 * square root twice; acos is CUDA's.
 */
#include <cuda_runtime.h>

#include <cstring>

#include "scatfield.h"

namespace {

constexpr int SF_WARPS = 4;
constexpr int SF_MAX_INTERACT = 1000000;

struct SfDev {
  TModel m;
  SfGeom g;
  const double *thet, *kext, *albedo, *F, *cum, *vis, *dirs;
  long long ncum;
  int mode;
  double Etot, Estar;
  long long nstar, nphot;
  unsigned long long key;
  double *SF;
  unsigned long long *stats;
};

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

__global__ void sf_opac_kernel(int ncell, int nc, int ncomp, int nlam, const double *comp_w, const double *Kabs_c,
                               const double *Ksca_c, const double *BB, const double *T, const double *dens,
                               const double *V, int l1, int l2, double w1, double w2, double *kabs, double *kext,
                               double *ksca, double *albedo, double *emis) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  sf_cell_opac(c, ncomp, nlam, comp_w, Kabs_c, Ksca_c, l1, l2, w1, w2, &kabs[c], &kext[c], &ksca[c], &albedo[c]);
  if (T)
    emis[c] = c >= nc ? sf_cell_emission(c, ncomp, nlam, comp_w, Kabs_c, BB, T[c], dens[c], V[c], l1, l2, w1, w2)
                      : 0.0;
}

__global__ void sf_mueller_kernel(long long n, int ncomp, int nlam, const double *comp_w, const double *Ksca_c,
                                  const double *F_c, const double *IF_c, int l1, int l2, double w1, double w2,
                                  const double *ksca, double *F) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = (int)(t / 1082), e = (int)(t % 1082);
  F[t] = sf_cell_mueller(c, e, ncomp, nlam, comp_w, Ksca_c, F_c, IF_c, l1, l2, w1, w2, ksca[c]);
}

__global__ void sf_exit_kernel(const __grid_constant__ TModel m, const double *kabs, int nexits, double *vis,
                               double *emis) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nt - 1;
  if (c >= m.ncell) return;
  const int i = c / nc, j = c % nc + 1;
  double v = 1.0;
  if (nexits > 0 && i >= 1) v = dm_exp(-sf_tauexit(m, kabs, i, j, nexits));
  vis[c] = v;
  emis[c] = emis[c] * v;
}

__device__ __forceinline__ size_t sf_base(const SfDev &d, int i, int j, int irg, int side) {
  return (((size_t)i * d.g.nsub + d.g.off[j - 1] + (irg - 1)) * 2 + side) * SF_NB;
}

/* the scattering-angle index (1..180) towards each observer direction and
 * the packet's Stokes Q in that direction's frame (TraceMono.f:1309-1337);
 * lanes take every 32nd direction */
__device__ void sf_directions(const SfDev &d, const TPkt &p, int lane, unsigned char *ia, double *q) {
  for (int k = lane; k < SF_NPHI; k += 32) {
    const double sx = d.dirs[3 * k], sy = d.dirs[3 * k + 1], sz = d.dirs[3 * k + 2];
    double c = (p.vx * sx + p.vy * sy) + p.vz * sz;
    c = fmin(1.0, fmax(-1.0, c));
    int a = (int)((180.0 * acos(c)) / TP_PI + 1.0);
    if (a > 180) a = 180;
    if (a < 1) a = 1;
    ia[k] = (unsigned char)(a - 1);
    double Qd = p.Q;
    if (p.pol) {
      double xn = p.vy * sz - p.vz * sy, yn = p.vz * sx - p.vx * sz, zn = p.vx * sy - p.vy * sx;
      const double r = sqrt((xn * xn + yn * yn) + zn * zn);
      if (r > 0.0) {
        xn = xn / r;
        yn = yn / r;
        zn = zn / r;
        TPkt t = p;
        tp_rotate_stokes(t, xn, yn, zn);
        Qd = t.Q;
      }
    }
    if (q) q[k] = Qd;
  }
}

/* the folded azimuth deposits of one segment (makescattfield,
 * TraceMono.f:1430-1497, and MakeStarScatter TraceMono.f:1695-1750): bin
 * i = 1..90 takes direction j0 + i - 1, bin 181 - i direction j0 + i - 1 for
 * i = 91..180 (directions wrapped into 1..180) */
__device__ void sf_fold(const SfDev &d, size_t base, const double *Fc, double x, double y, double E, double vAU,
                        const unsigned char *ia, const double *q, bool withQ, int lane) {
  const double rho = sqrt(x * x + y * y);
  double phi0 = rho > 0.0 ? (180.0 * acos(x / rho)) / TP_PI : 0.0;
  if (y < 0.0) phi0 = 360.0 - phi0;
  const double phi = 180.0 / (double)(float)SF_NPHI;
  const int j0 = (int)(((double)(float)SF_NPHI * (phi + phi0)) / 360.0);
  for (int k = lane; k < SF_NPHI; k += 32) {
    int j = j0 + k;
    if (j < 1) j = j + SF_NPHI;
    if (j > SF_NPHI) j = j - SF_NPHI;
    const int a = ia[j - 1];
    const double sI = withQ ? Fc[a] * E + Fc[180 + a] * q[j - 1] : Fc[a] * E;
    const int bin = k < SF_NPHI / 2 ? k + 1 : SF_NPHI - k;
    atomicAdd(&d.SF[base + bin], sI * vAU);
  }
}

/* the start of a packet on the stellar surface, moving outward
 * (TraceMono.f:1140-1170, 1613-1637); false when |z|/R0 sits exactly on a
 * theta edge (the reference draws again there).  The sub-cell takes the
 * polar angle of |z|/R0 (byct, MakeStarScatter) or of |z|/r (emitposition). */
__device__ bool sf_star_start(const SfDev &d, px_stream *r, TPkt &p, int *irg, bool byct) {
  const TModel &m = d.m;
  const double R0 = m.R[0];
  tp_randomdirection(r, &p.x, &p.y, &p.z);
  p.x = R0 * p.x;
  p.y = R0 * p.y;
  p.z = R0 * p.z;
  tp_randomdirection(r, &p.vx, &p.vy, &p.vz);
  const double inp = (p.x * p.vx + p.y * p.vy) + p.z * p.vz;
  if (inp < 0.0) {
    p.vx = -p.vx;
    p.vy = -p.vy;
    p.vz = -p.vz;
  }
  p.edgeNr = 1;
  p.onEdge = 1;
  const double ct = fabs(p.z) / R0;
  for (int j = 1; j <= m.nt - 1; ++j)
    if (ct < m.Theta[j - 1] && ct > m.Theta[j]) {
      p.i = 0;
      p.j = j;
      *irg = sf_irg(d.g, d.thet, j, acos(byct ? ct : fabs(p.z) / sqrt((p.x * p.x + p.y * p.y) + p.z * p.z)));
      return true;
    }
  return false;
}

/* emitposition (TraceMono.f:1124-1290) without the interstellar field and
 * the inner gas disk: starlight with probability Estar / Etot, else a
 * point in the cell chosen by the weighted emission; false when 1000
 * draws found no start */
__device__ bool sf_emit(const SfDev &d, px_stream *r, TPkt &p, int *irg) {
  const TModel &m = d.m;
  const int nc = m.nt - 1;
  for (int tries = 0; tries < 1000; ++tries) {
    p.pol = 0;
    const double Etot = d.Etot;
    double Er = Etot * px_next(r);
    if (Er < d.Estar) {
      p.E = Etot;
      p.scatt = 0;
      if (sf_star_start(d, r, p, irg, false)) return true;
      continue;
    }
    p.scatt = 1;
    Er = Er - d.Estar;
    long long lo = 0, hi = d.ncum; /* first cell whose running sum exceeds Er */
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (Er < d.cum[mid])
        hi = mid;
      else
        lo = mid + 1;
    }
    if (lo >= d.ncum) continue;
    const int i = 1 + (int)(lo / nc), j = 1 + (int)(lo % nc);
    double Rad = px_next(r);
    Rad = sqrt(m.R[i] * m.R[i] * Rad + m.R[i + 1] * m.R[i + 1] * (1.0 - Rad));
    double Th = px_next(r);
    Th = m.Theta[j - 1] * Th + m.Theta[j] * (1.0 - Th);
    p.z = Rad * Th;
    if (px_next(r) < 0.5) p.z = -p.z;
    const double phi = (px_next(r) * TP_PI) * 2.0;
    p.x = (Rad * sqrt(1.0 - Th * Th)) * dm_sin(phi);
    p.y = (Rad * sqrt(1.0 - Th * Th)) * dm_cos(phi);
    tp_randomdirection(r, &p.vx, &p.vy, &p.vz);
    p.i = i;
    p.j = j;
    *irg = sf_irg(d.g, d.thet, j, acos(fabs(p.z) / sqrt((p.x * p.x + p.y * p.y) + p.z * p.z)));
    p.onEdge = 0;
    p.edgeNr = 0;
    p.E = Etot / d.vis[(size_t)i * nc + (j - 1)];
    return true;
  }
  return false;
}

__global__ void __launch_bounds__(32 * SF_WARPS) sf_star_kernel(const __grid_constant__ SfDev d) {
  __shared__ unsigned char s_ia[SF_WARPS][SF_NPHI];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long w = (long long)blockIdx.x * SF_WARPS + wib;
  if (w >= d.nstar) return;
  const TModel &m = d.m;
  const int nc = m.nt - 1;
  px_stream r;
  px_init(&r, d.key, (uint64_t)w);
  TPkt p;
  memset(&p, 0, sizeof p);
  int irg = 1;
  p.E = d.Estar / (double)(float)d.nstar;
  p.scatt = 0;
  if (!sf_star_start(d, &r, p, &irg, true)) {
    /* |z|/R0 on a theta edge: the row below it */
    const double ct = fabs(p.z) / m.R[0];
    p.i = 0;
    p.j = 1;
    for (int j = 1; j <= nc; ++j)
      if (ct <= m.Theta[j - 1] && ct >= m.Theta[j]) {
        p.j = j;
        break;
      }
    irg = sf_irg(d.g, d.thet, p.j, acos(ct));
  }
  unsigned char *ia = s_ia[wib];
  if (d.mode == 2) sf_directions(d, p, lane, ia, nullptr);
  __syncwarp();
  for (int n = 0;; ++n) {
    double v;
    int inext, jnext, irgn;
    if (n >= (1 << 20) || sf_trace2edge_rg(m, d.g, p, irg, &v, &inext, &jnext, &irgn) != 0) {
      if (lane == 0) atomicAdd(&d.stats[0], 1ull);
      break;
    }
    const size_t c = (size_t)p.i * nc + (p.j - 1);
    const double tau = (m.dens[c] * d.kext[c]) * TP_AU;
    const double w1 = (tau * v > 1e-5) ? (1.0 - dm_exp(-tau * v)) / tau : v;
    if (d.mode == 1) {
      const size_t b = sf_base(d, p.i, p.j, 1, 0);
      if (lane == 0) {
        atomicAdd(&d.SF[b], ((p.E * w1) * TP_AU) / 2.0);
        atomicAdd(&d.SF[b + SF_NB], ((p.E * w1) * TP_AU) / 2.0);
      }
    } else {
      const double x = p.x + (p.vx * v) / 2.0, y = p.y + (p.vy * v) / 2.0;
      const int ir = irg < 1 ? 1 : irg;
      const size_t b = sf_base(d, p.i, p.j, ir, p.z > 0.0 ? 0 : 1);
      if (lane == 0) atomicAdd(&d.SF[b], (p.E * w1) * TP_AU);
      sf_fold(d, b, d.F + c * 1082, x, y, p.E, (v * TP_AU) / 2.0, ia, nullptr, false, lane);
    }
    p.E = p.E * dm_exp(-tau * v);
    p.x = p.x + p.vx * v;
    p.y = p.y + p.vy * v;
    p.z = p.z + p.vz * v;
    p.onEdge = 1;
    if (inext >= m.nr || inext < 0) break;
    p.i = inext;
    p.j = jnext;
    irg = irgn;
  }
}

__global__ void __launch_bounds__(32 * SF_WARPS) sf_mc_kernel(const __grid_constant__ SfDev d) {
  __shared__ unsigned char s_ia[SF_WARPS][SF_NPHI];
  __shared__ double s_q[SF_WARPS][SF_NPHI];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long w = (long long)blockIdx.x * SF_WARPS + wib;
  if (w >= d.nphot) return;
  const TModel &m = d.m;
  const int nc = m.nt - 1;
  unsigned char *ia = s_ia[wib];
  double *q = s_q[wib];
  px_stream r;
  px_init(&r, d.key, (uint64_t)(d.nstar + w));
  TPkt p;
  memset(&p, 0, sizeof p);
  int irg = 1;
  if (!sf_emit(d, &r, p, &irg)) {
    if (lane == 0) atomicAdd(&d.stats[2], 1ull);
    return;
  }
  p.E = p.E / (double)(float)d.nphot;
  if (d.mode == 2) {
    p.pol = 0;
    p.Q = 0.0;
    p.U = 0.0;
    p.V = 0.0;
    double x, y, z;
    if (p.vz != 1.0) {
      x = -p.vy;
      y = p.vx;
      z = 0.0;
    } else {
      x = 1.0;
      y = 0.0;
      z = 0.0;
    }
    const double rr = sqrt((x * x + y * y) + z * z);
    p.Sx = x / rr;
    p.Sy = y / rr;
    p.Sz = z / rr;
  }
  const int maxv = (m.nr + m.nt + 360) * 2;
  for (int nint = 0;; ++nint) {
    const double tau0 = -dm_log(px_next(&r));
    __syncwarp();
    const bool dirs = d.mode == 2 && p.scatt;
    if (dirs) sf_directions(d, p, lane, ia, q);
    __syncwarp();
    /* trace2dmono, TraceMono.f:1339-1411 */
    double tau = 0.0;
    bool escape = false, interact = false;
    for (int nv = 1;; ++nv) {
      double v;
      int inext, jnext, irgn;
      if (nv > maxv) {
        escape = true;
        break;
      }
      if (sf_trace2edge_rg(m, d.g, p, irg, &v, &inext, &jnext, &irgn) != 0) {
        if (lane == 0) atomicAdd(&d.stats[0], 1ull);
        escape = true;
        break;
      }
      const size_t c = (size_t)p.i * nc + (p.j - 1);
      const double tau1 = ((v * m.dens[c]) * d.kext[c]) * TP_AU;
      if (tau + tau1 > tau0) {
        v = (v * (tau0 - tau)) / tau1;
        interact = true;
      }
      if (p.scatt) { /* makescattfield */
        if (d.mode == 1) {
          const size_t b = sf_base(d, p.i, p.j, 1, 0);
          if (lane == 0) {
            atomicAdd(&d.SF[b], ((p.E * v) * TP_AU) / 2.0);
            atomicAdd(&d.SF[b + SF_NB], ((p.E * v) * TP_AU) / 2.0);
          }
        } else {
          const double x = p.x + (p.vx * v) / 2.0, y = p.y + (p.vy * v) / 2.0;
          const int ir = irg < 1 ? 1 : irg;
          const size_t b = sf_base(d, p.i, p.j, ir, p.z > 0.0 ? 0 : 1);
          if (lane == 0) atomicAdd(&d.SF[b], (p.E * v) * TP_AU);
          sf_fold(d, b, d.F + c * 1082, x, y, p.E, (v * TP_AU) / 2.0, ia, q, true, lane);
        }
      }
      p.x = p.x + p.vx * v;
      p.y = p.y + p.vy * v;
      p.z = p.z + p.vz * v;
      if (interact) {
        p.onEdge = 0;
        break;
      }
      p.onEdge = 1;
      tau = tau + tau1;
      if (inext >= m.nr || inext < 0) {
        escape = true;
        break;
      }
      p.i = inext;
      p.j = jnext;
      irg = irgn;
    }
    if (escape) break;
    /* the albedo roulette and the scattering, TraceMono.f:859-878 */
    const size_t c = (size_t)p.i * nc + (p.j - 1);
    const double alb = d.albedo[c];
    const double fstop = sqrt(sqrt(alb));
    if (!(fstop > 0.0)) break;
    const double fact = alb / fstop;
    p.E = p.E * fact;
    p.Q = p.Q * fact;
    p.U = p.U * fact;
    p.V = p.V * fact;
    if (px_next(&r) > fstop) break;
    if (nint >= SF_MAX_INTERACT) {
      if (lane == 0) atomicAdd(&d.stats[1], 1ull);
      break;
    }
    p.scatt = 1;
    if (d.mode == 1)
      tp_randomdirection(&r, &p.vx, &p.vy, &p.vz);
    else
      tp_scatangle(m, &r, p, d.F + c * 1082, d.F + c * 1082 + 1080);
  }
}

/* the observer directions of an inclination (TracePath, TraceMono.f:2058-2075) */
void sf_observer_dirs(double angle, double *dirs) {
  for (int i = 1; i <= SF_NPHI; ++i) {
    const double phi = (TP_PI * ((double)(float)i - 0.5)) / ((double)(float)SF_NPHI / 2.0);
    double x = 0.0, y = 0.0, z = 1.0;
    tp_rotate(&x, &y, &z, 0.0, 1.0, 0.0, angle);
    tp_rotate(&x, &y, &z, 0.0, 0.0, 1.0, phi);
    const double r = sqrt((x * x + y * y) + z * z);
    dirs[3 * (i - 1)] = x / r;
    dirs[3 * (i - 1) + 1] = y / r;
    dirs[3 * (i - 1) + 2] = z / r;
  }
}

}  // namespace

SfState::~SfState() {
  for (void *p : owned) cudaFree(p);
}

bool SfState::fail(cudaError_t e, const char *what) {
  err = std::string("scattering field: ") + what + ": " + cudaGetErrorString(e);
  return false;
}

template <class T>
bool SfState::alloc(T **p, size_t n) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, sizeof(T) * (n ? n : 1));
  if (e != cudaSuccess) return fail(e, "allocation");
  owned.push_back(q);
  *p = (T *)q;
  return true;
}

bool SfState::init(mcg_ctx *c, double ang, const SfOpts &opts, const double *Theta_h) {
  ctx = c;
  st = c->stream;
  o = opts;
  angle = ang;
  const DevModel &m = c->model;
  mode = 0;
  if ((o.nphot > 0 || o.nstar > 0) && m.scattering) mode = m.scat_how == 2 ? 2 : (m.scat_how == 1 ? 1 : 0);
  if (!mode) return true;
  const int nt = m.nt, nc = nt - 1;
  std::vector<double> th(nt);
  for (int j = 0; j < nt; ++j) th[j] = acos(Theta_h[j]);
  th[0] = 0.0;
  th[nt - 1] = TP_PI / 2.0;
  sf_geom_build(nt, th.data(), Theta_h, mode == 2, &gh);
  int *dn, *doff;
  double *dtr, *dfr;
  if (!alloc(&dn, nc) || !alloc(&doff, nc) || !alloc(&dtr, gh.thetrg.size()) || !alloc(&dfr, gh.fracirg.size()) ||
      !alloc(&thet, nt))
    return false;
  cudaError_t e = cudaMemcpyAsync(dn, gh.nrg.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(doff, gh.off.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dtr, gh.thetrg.data(), sizeof(double) * gh.thetrg.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dfr, gh.fracirg.data(), sizeof(double) * gh.fracirg.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(thet, th.data(), sizeof(double) * nt, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(e, "upload");
  g.nsub = gh.nsub;
  g.nrg = dn;
  g.off = doff;
  g.thetrg = dtr;
  g.fracirg = dfr;
  const size_t ncell = m.ncell;
  if (!alloc(&kabs, ncell) || !alloc(&kext, ncell) || !alloc(&ksca, ncell) || !alloc(&albedo, ncell) ||
      !alloc(&emis, ncell) || !alloc(&vis, ncell) || !alloc(&cum, ncell) || !alloc(&dirs, 3 * SF_NPHI) ||
      !alloc(&stats, 3))
    return false;
  if (mode == 2 && !alloc(&F, ncell * 1082)) return false;
  std::vector<double> hd(3 * SF_NPHI, 0.0);
  if (mode == 2) sf_observer_dirs(angle, hd.data());
  e = cudaMemcpyAsync(dirs, hd.data(), sizeof(double) * hd.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * 3, st);
  if (e != cudaSuccess) return fail(e, "upload");
  field_len = (size_t)m.nr * gh.nsub * 2 * SF_NB;
  return true;
}

bool SfState::albedo_at(double lam0) {
  const DevModel &m = ctx->model;
  int l1, l2;
  double w1, w2;
  sf_lam(m.nlam, m.lam_h.data(), lam0, &l1, &l2, &w1, &w2);
  /* TraceFlux's opacities at lam0 */
  sf_opac_kernel<<<nblk(m.ncell, 128), 128, 0, st>>>(m.ncell, m.nt - 1, m.ncomp, m.nlam, m.comp_w, m.Kabs_c, m.Ksca_c,
                                                     m.BB, nullptr, m.dens, m.V, l1, l2, w1, w2, kabs, kext, ksca,
                                                     albedo, emis);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? true : fail(e, "opacity kernel");
}

bool SfState::compute(double lam0, const double *T, double *out) {
  const DevModel &m = ctx->model;
  const int nc = m.nt - 1;
  int l1, l2;
  double w1, w2;
  sf_lam(m.nlam, m.lam_h.data(), lam0, &l1, &l2, &w1, &w2);
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * field_len, st);
  if (e != cudaSuccess) return fail(e, "memset");
  sf_opac_kernel<<<nblk(m.ncell, 128), 128, 0, st>>>(m.ncell, nc, m.ncomp, m.nlam, m.comp_w, m.Kabs_c, m.Ksca_c, m.BB,
                                                     T, m.dens, m.V, l1, l2, w1, w2, kabs, kext, ksca, albedo, emis);
  if (mode == 2) {
    const long long n = (long long)m.ncell * 1082;
    sf_mueller_kernel<<<nblk(n, 256), 256, 0, st>>>(n, m.ncomp, m.nlam, m.comp_w, m.Ksca_c, m.F_c, m.IF_c, l1, l2, w1,
                                                    w2, ksca, F);
  }
  TModel tm;
  memset(&tm, 0, sizeof tm);
  tm.nr = m.nr;
  tm.nt = m.nt;
  tm.nc = m.nc;
  tm.ncell = m.ncell;
  tm.scat_how = m.scat_how;
  tm.R = m.R;
  tm.Theta = m.Theta;
  tm.dens = m.dens;
  tm.sinthet = m.sinthet;
  tm.cos2phi = m.cos2phi;
  tm.sin2phi = m.sin2phi;
  sf_exit_kernel<<<nblk(m.ncell, 64), 64, 0, st>>>(tm, kabs, o.nexits, vis, emis);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(e, "cell kernels");
  /* EmissionDistribution's running sum over i = 1..nR-1, j = 1..nTheta-1 */
  std::vector<double> he(m.ncell);
  e = cudaMemcpyAsync(he.data(), emis, sizeof(double) * m.ncell, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(e, "emission");
  const long long ncum = (long long)(m.nr - 1) * nc;
  std::vector<double> hc((size_t)(ncum > 0 ? ncum : 1));
  double Et = 0.0;
  for (long long k = 0; k < ncum; ++k) {
    Et = Et + he[(size_t)nc + k];
    hc[k] = Et;
  }
  e = cudaMemcpyAsync(cum, hc.data(), sizeof(double) * hc.size(), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(e, "upload");
  SfDev d;
  memset(&d, 0, sizeof d);
  d.m = tm;
  d.g = g;
  d.thet = thet;
  d.kext = kext;
  d.albedo = albedo;
  d.F = F;
  d.cum = cum;
  d.vis = vis;
  d.dirs = dirs;
  d.ncum = ncum;
  d.mode = mode;
  d.Estar = m.Fstar_h[l1] * w1 + m.Fstar_h[l2] * w2;
  d.Etot = Et + d.Estar;
  d.nstar = o.nstar;
  d.nphot = o.nphot;
  d.key = (unsigned long long)(o.seed + nfields);
  d.SF = out;
  d.stats = stats;
  ++nfields;
  if (o.nstar > 0) sf_star_kernel<<<nblk(o.nstar, SF_WARPS), 32 * SF_WARPS, 0, st>>>(d);
  if (o.nphot > 0 && d.Etot > 0.0) sf_mc_kernel<<<nblk(o.nphot, SF_WARPS), 32 * SF_WARPS, 0, st>>>(d);
  e = cudaGetLastError();
  return e == cudaSuccess ? true : fail(e, "packet kernels");
}

bool SfState::prepare(double lam0, const double *T, const double **f1, const double **f2, double *w1, double *w2) {
  const DevModel &m = ctx->model;
  if (mode == 2) {
    if (!field && !alloc(&field, field_len)) return false;
    if (!compute(lam0, T, field)) return false;
    *f1 = field;
    *f2 = field;
    *w1 = 1.0;
    *w2 = 0.0;
    return true;
  }
  int l1, l2;
  sf_lam(m.nlam, m.lam_h.data(), lam0, &l1, &l2, w1, w2);
  for (int l : {l1, l2}) {
    if (iso.count(l)) continue;
    double *buf;
    if (!alloc(&buf, field_len)) return false;
    if (!compute(m.lam_h[l], T, buf)) return false;
    iso[l] = buf;
  }
  *f1 = iso[l1];
  *f2 = iso[l2];
  return albedo_at(lam0);
}
