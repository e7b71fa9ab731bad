/*
 * transport_core.cuh -- the photon-packet loop of MCMax (MCRadiation.f,
 * Radiation.f, RandomWalk.f) as per-packet code for one GPU thread, in FP64.
 *
 * One thread owns one packet from emission to escape; when it is done it
 * takes the next packet id from a global counter (persistent threads that
 * refill their lane instead of idling until the slowest packet of the warp
 * finishes).  Per-cell accumulators (EJv, EJv2, Eabs, Ni) are updated with
 * atomics; the Bjorkman-Wood temperature of a cell is a pure function of its
 * absorbed energy, so a packet derives T0 and T1 from the Eabs values before
 * and after its own atomic increment and re-emits exactly the energy it
 * added, whatever the interleaving with other packets.
 *
 * The source compiles for the device and, unchanged, for the host (one
 * thread, atomics become plain updates) so a run can be replayed on the CPU.
 * With one thread the packet order is the reference's serial order and the
 * result matches the CPU oracle bit for bit (FP64 path, --fmad=false,
 * detmath.h transcendentals).
 *
 * Reference map:
 *   tp_run_packet      MCRadiation.f:320-648 (star emission :355-382,
 *                      escape/SED :576-646, overflow :568-571)
 *   tp_trace2d         MCRadiation.f:901-1141
 *   tp_trace2edge      MCRadiation.f:1150-1272, hitR/hitT/hitTsame :1274-1355
 *   tp_interact        Radiation.f:41-315 (thermal contact)
 *   tp_scatangle       Radiation.f:381-495, RotateStokes :506-534
 *   tp_emit_*          Radiation.f:940-1001, randomdirection :1007-1024
 *   tp_random_walk     RandomWalk.f:15-147, hunt Subroutines.f:2086-2132
 *   tp_tinv            increaseT/determineT, Radiation.f:537-702
 */
#ifndef MCMAX_TRANSPORT_CORE_CUH
#define MCMAX_TRANSPORT_CORE_CUH

#include <stdint.h>

#include "detmath.h"
#include "philox.h"

#if defined(__CUDACC__)
#define TP_SFN static __host__ __device__ __forceinline__
#define TP_FN __host__ __device__ __forceinline__
#define TP_NOINLINE static __host__ __device__ __noinline__
#else
#define TP_SFN static inline
#define TP_FN static inline
#define TP_NOINLINE static
#endif

#define TP_TMAX 10000
#define TP_TT (TP_TMAX + 1)
/* the reference declares AU real*8 but gives it a default-real literal,
 * parameter(AU=1.49598e13) (Modules.f:4,8): its value is the single-precision
 * number nearest 1.49598e13, widened */
#define TP_AU ((double)1.49598e13f)
#define TP_PI 3.14159265358979323846
#define TP_NY 1000
#define TP_NANG 30

/* counters, same slots as mcg_result.counters */
enum {
  TC_EMIT = 0, TC_INTERACT, TC_ABSORB, TC_SCATTER, TC_RWSTEP, TC_HITSTAR, TC_ABANDON,
  TC_OVERFLOW, TC_CROSS, TC_ESCAPE, TC_AVGMAT, TC_GEOFAIL, TC_N = 16
};

/* model tables, device (or host) pointers */
struct TModel {
  int nr, nt, nc, ncell, nlam, ncomp;
  int scattering, scat_how, uniform_mix, rw;
  double factRW, R0, Lstar, Epkt;
  int64_t nphot, maxinteract;
  int64_t pid0;   /* packet-id offset of this run (nruns > 1) */
  double nruns_d; /* real(nruns), divides the SED contributions */
  uint64_t seed;
  const double *R, *Theta, *SinTheta, *dens, *mass;
  const double *nu, *dnu_half, *BB, *star_cdf, *wlam;
  const double *KabsTot, *KscaTot, *KpCell, *emit_cdf;
  const double *comp_w, *Ksca_c, *F_c, *IF_c;
  const double *sinthet, *cos2phi, *sin2phi;
  const double *KDext, *KDabs, *rw_y, *rw_phi;
  const int *kd_index;
  const unsigned char *thick;
  double maxruntime; /* seconds; > 0: the run-time limit of MCRadiation.f:323-342 */
  int t4single;      /* 1: the temperature interpolation's i^4 in single precision, as the reference */
};

/* accumulators */
struct TAcc {
  /* per-cell arrays hold nruns blocks of ncell entries: the independent
   * sub-runs of the reference's nruns loop (MCRadiation.f:269-316) run
   * concurrently, packet p belonging to run p / run_packets */
  double *EJv, *EJv2, *Eabs, *T;
  int *Ni, *lastphot, *kp_hint;
  double *spec, *scatspec;
  int *ispec;
  unsigned long long *counters;
  double *tautot;
  unsigned long long *next;
  int64_t run_packets;
  int ncell;
  /* progress marks: globaltimer when 50/90/99/99.9/100 % of the packets are
   * done, [5] = kernel start */
  unsigned long long *done, *tmark;
  unsigned long long thresh[5];
  int *Nabs;                /* absorption events per cell (may be null) */
  unsigned long long *stop; /* maxruntime: [0] packets started when the run
                               stopped (0: running), [1] elapsed ns then */
};

/* accumulators of the run that packet pid belongs to */
TP_FN TAcc tp_run_acc(const TAcc &A, int64_t pid) {
  TAcc R = A;
  const size_t off = (size_t)(pid / A.run_packets) * (size_t)A.ncell;
  R.EJv += off;
  R.EJv2 += off;
  R.Eabs += off;
  R.T += off;
  R.Ni += off;
  R.lastphot += off;
  R.kp_hint += off;
  if (R.Nabs) R.Nabs += off;
  return R;
}

TP_FN unsigned long long tp_globaltimer() {
#if defined(__CUDA_ARCH__)
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
#else
  return 0ULL;
#endif
}

/* count a finished packet; record the progress marks */
TP_FN void tp_packet_done(const TAcc &A) {
#if defined(__CUDA_ARCH__)
  const unsigned long long d = atomicAdd(A.done, 1ULL) + 1ULL;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    if (d == A.thresh[k]) A.tmark[k] = tp_globaltimer();
#else
  (void)A;
#endif
}

/* ------------------------------------------------------------- atomics */
TP_FN double tp_add(double *p, double v) {
#if defined(__CUDA_ARCH__)
  return atomicAdd(p, v);
#else
  double o = *p;
  *p = o + v;
  return o;
#endif
}
/* The run-time limit of MCRadiation.f:323-342, checked when the run's
 * packet k (0-based) is about to start, t0 the caller's start time
 * (globaltimer, ns): the run stops when more than maxruntime seconds have
 * passed, or when more than a tenth of the packets have started and the run
 * projects to more than 5 maxruntime -- in both cases only with under 90 %
 * of the packets started.  The first thread to see it records the packet
 * count and the elapsed time; returns 1 when the run is stopping. */
TP_FN int tp_runtime_stop(const TAcc &A, double maxruntime, int64_t nphot, unsigned long long k,
                          unsigned long long t0) {
#if defined(__CUDA_ARCH__)
  if (!(maxruntime > 0.0) || nphot <= 10 || !A.stop) return 0;
  if (*(volatile unsigned long long *)A.stop) return 1;
  const double t = (double)(tp_globaltimer() - t0) * 1e-9;
  const unsigned long long i = k + 1ULL;
  const double di = (double)i, dn = (double)nphot;
  if ((t > maxruntime || (i > (unsigned long long)(nphot / 10) && t * dn / di > 5.0 * maxruntime)) && di / dn < 0.9) {
    if (atomicCAS(A.stop, 0ULL, i) == 0ULL) A.stop[1] = (unsigned long long)(t * 1e9);
    return 1;
  }
  return 0;
#else
  (void)A; (void)maxruntime; (void)nphot; (void)k; (void)t0;
  return 0;
#endif
}

TP_FN void tp_addi(int *p, int v) {
#if defined(__CUDA_ARCH__)
  atomicAdd(p, v);
#else
  *p += v;
#endif
}
TP_FN int tp_exch(int *p, int v) {
#if defined(__CUDA_ARCH__)
  return atomicExch(p, v);
#else
  int o = *p;
  *p = v;
  return o;
#endif
}

/* ------------------------------------------------------------- packet */
struct TPkt {
  double x, y, z, vx, vy, vz;
  double E, Q, U, V, Sx, Sy, Sz;
  double wl1, wl2;
  double nEJv;
  int ilam1, ilam2, i, j, edgeNr;
  int onEdge, scatt, pol;
  int pid1; /* packet number + 1 (lastphotnr) */
};

struct TLocal {
  unsigned int cnt[TC_N]; /* per-thread event counts, flushed at exit */
  double tautot;
};

TP_FN double tp_rnd(px_stream *r) { return px_next(r); }

TP_FN void tp_randomdirection(px_stream *r, double *x, double *y, double *z) {
  double rr;
  for (;;) {
    *x = 2.0 * tp_rnd(r) - 1.0;
    *y = 2.0 * tp_rnd(r) - 1.0;
    *z = 2.0 * tp_rnd(r) - 1.0;
    rr = ((*x) * (*x) + (*y) * (*y)) + (*z) * (*z);
    if (!(rr > 1.0)) break;
  }
  rr = sqrt(rr);
  *x = *x / rr;
  *y = *y / rr;
  *z = *z / rr;
}

TP_FN void tp_set_s(TPkt &p) {
  double x = -p.vy, y = p.vx, z = 0.0;
  double r = sqrt((x * x + y * y) + z * z);
  p.Sx = x / r;
  p.Sy = y / r;
  p.Sz = z / r;
}

/* first index i in [0,n) with cdf[i] >= v, or n */
TP_FN int tp_lower_bound(const double *cdf, int n, double v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (cdf[mid] >= v)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

/* wavelength pick from a cumulative table (identical to the reference's
 * linear scan because the cumulative values are built in the same order) */
TP_FN void tp_pick_cdf(const TModel &m, TPkt &p, const double *cdf, double Lr) {
  const int n = m.nlam - 1;
  int i = tp_lower_bound(cdf, n, Lr);
  if (i < n) {
    double Lt = cdf[i];
    double Ltold = i > 0 ? cdf[i - 1] : 0.0;
    double d = Lt - Ltold;
    p.wl1 = d != 0.0 ? (Lr - Ltold) / d : 1.0;
    p.wl2 = 1.0 - p.wl1;
    p.ilam1 = i;
    p.ilam2 = i + 1;
  } else {
    p.wl1 = 0.0;
    p.wl2 = 1.0;
    p.ilam1 = m.nlam - 2;
    p.ilam2 = m.nlam - 1;
  }
}

/* direction + reference axis of a fresh emission (start of emit) */
TP_FN void tp_emit_dir(px_stream *r, TPkt &p, TLocal &L) {
  L.cnt[TC_EMIT]++;
  tp_randomdirection(r, &p.vx, &p.vy, &p.vz);
  p.scatt = 0;
  p.pol = 0;
  tp_set_s(p);
}

/* ------------------------------------------------------------- geometry */
TP_FN int tp_hitR(double Rad, double r, double b, double *v) {
  int hit = 0;
  *v = 1e200;
  double cc = r - Rad;
  double discr = b * b - 4.0 * cc;
  if (discr >= 0.0) {
    discr = sqrt(discr);
    double q = (b > 0.0) ? -0.5 * (b + discr) : -0.5 * (b - discr);
    double vr1 = q, vr2 = cc / q;
    if (vr1 > 0.0) {
      *v = vr1;
      hit = 1;
    }
    if (vr2 > 0.0 && vr2 < *v) {
      *v = vr2;
      hit = 1;
    }
  }
  return hit;
}

TP_FN int tp_hitT(const TPkt &p, double Thet, double r, double b, double *v) {
  int hit = 0;
  *v = 1e200;
  double at = Thet - p.vz * p.vz;
  double bt = Thet * b - (2.0 * p.z) * p.vz;
  double ct = Thet * r - p.z * p.z;
  double discr = bt * bt - (4.0 * at) * ct;
  if (discr >= 0.0) {
    discr = sqrt(discr);
    double q = (bt > 0.0) ? -0.5 * (bt + discr) : -0.5 * (bt - discr);
    double vt1 = q / at, vt2 = ct / q;
    if (vt1 > 0.0) {
      *v = vt1;
      hit = 1;
    }
    if (vt2 > 0.0 && vt2 < *v) {
      *v = vt2;
      hit = 1;
    }
  }
  return hit;
}

TP_FN int tp_hitTsame(const TPkt &p, double Thet, double b, double *v) {
  double bt = Thet * b - (2.0 * p.z) * p.vz;
  double at = Thet - p.vz * p.vz;
  *v = (-bt) / at;
  return *v > 0.0;
}

/* distance to the next cell boundary; 1 when nothing can be hit */
TP_FN int tp_trace2edge(const TModel &m, TPkt &p, double *v, int *inext, int *jnext) {
  const int nt = m.nt;
  double r = (p.x * p.x + p.y * p.y) + p.z * p.z;
  double Ra = m.R[p.i], Rb = m.R[p.i + 1];
  double Ta = m.Theta[p.j - 1], Tb = m.Theta[p.j];
  double R1 = Ra * Ra, R2 = Rb * Rb, T1 = Ta * Ta, T2 = Tb * Tb;
  double b = 2.0 * ((p.x * p.vx + p.y * p.vy) + p.z * p.vz);
  int hR1, hR2, hT1, hT2;
  double vR1, vR2, vT1, vT2;
  if (!p.onEdge) {
    hR1 = tp_hitR(R1, r, b, &vR1);
    hR2 = tp_hitR(R2, r, b, &vR2);
    hT1 = tp_hitT(p, T1, r, b, &vT1);
    hT2 = tp_hitT(p, T2, r, b, &vT2);
  } else if (p.edgeNr == 1) {
    hR1 = 0;
    vR1 = 1e200;
    hR2 = tp_hitR(R2, r, b, &vR2);
    hT1 = tp_hitT(p, T1, r, b, &vT1);
    hT2 = tp_hitT(p, T2, r, b, &vT2);
  } else if (p.edgeNr == 2) {
    hR1 = tp_hitR(R1, r, b, &vR1);
    hR2 = 1;
    vR2 = -b;
    hT1 = tp_hitT(p, T1, r, b, &vT1);
    hT2 = tp_hitT(p, T2, r, b, &vT2);
  } else if (p.edgeNr == 3) {
    hR1 = tp_hitR(R1, r, b, &vR1);
    hR2 = tp_hitR(R2, r, b, &vR2);
    hT1 = 0;
    vT1 = 1e200;
    if (p.j != nt - 1) {
      hT2 = tp_hitT(p, T2, r, b, &vT2);
    } else {
      vT2 = -p.z / p.vz;
      hT2 = vT2 > 0.0;
    }
  } else {
    hR1 = tp_hitR(R1, r, b, &vR1);
    hR2 = tp_hitR(R2, r, b, &vR2);
    if (p.j != 1) {
      hT1 = tp_hitT(p, T1, r, b, &vT1);
    } else {
      hT1 = 0;
      vT1 = 1e200;
    }
    if (p.j != nt - 1) {
      hT2 = tp_hitTsame(p, T2, b, &vT2);
    } else {
      hT2 = 0;
      vT2 = 1e200;
    }
  }
  if (!hR1 && !hR2 && !hT1 && !hT2) {
    hR1 = tp_hitR(R1, r, b, &vR1);
    hR2 = tp_hitR(R2, r, b, &vR2);
    hT1 = tp_hitT(p, T1, r, b, &vT1);
    hT2 = tp_hitT(p, T2, r, b, &vT2);
    if (!hR1 && !hR2 && !hT1 && !hT2) return 1;
  }
  *v = 1e200;
  *inext = p.i;
  *jnext = p.j;
  if (hR1 && vR1 < *v) {
    *v = vR1;
    *inext = p.i - 1;
    *jnext = p.j;
    p.edgeNr = 2;
  }
  if (hR2 && vR2 < *v) {
    *v = vR2;
    *inext = p.i + 1;
    *jnext = p.j;
    p.edgeNr = 1;
  }
  if (hT1 && vT1 < *v) {
    *v = vT1;
    *inext = p.i;
    *jnext = p.j - 1;
    p.edgeNr = 4;
  }
  if (hT2 && vT2 < *v) {
    *v = vT2;
    *inext = p.i;
    *jnext = p.j + 1;
    p.edgeNr = 3;
  }
  if (*jnext == nt) {
    *jnext = nt - 1;
    p.edgeNr = 4;
  }
  if (*jnext == 0) {
    *jnext = 1;
    p.edgeNr = 3;
  }
  return 0;
}

TP_FN void tp_rotate(double *x, double *y, double *z, double u, double v, double w, double theta) {
  double cost = dm_cos(theta), sint = dm_sin(theta);
  double u2 = u * u, v2 = v * v, w2 = w * w;
  double inp = (*x * u + *y * v) + *z * w;
  double y1 = (u * inp + (*x * (v2 + w2) - u * (v * *y + w * *z)) * cost) + (v * *z - w * *y) * sint;
  double y2 = (v * inp + (*y * (u2 + w2) - v * (u * *x + w * *z)) * cost) + (w * *x - u * *z) * sint;
  double y3 = (w * inp + (*z * (u2 + v2) - w * (u * *x + v * *y)) * cost) + (u * *y - v * *x) * sint;
  *x = y1;
  *y = y2;
  *z = y3;
}

TP_FN void tp_rotate_stokes(TPkt &p, double x, double y, double z) {
  double P = (p.U / p.E) * (p.U / p.E) + (p.Q / p.E) * (p.Q / p.E);
  if (P == 0.0) return;
  double cost = (p.Sx * x + p.Sy * y) + p.Sz * z;
  double sint = (x - (p.Sx * (p.vy * p.vy + p.vz * p.vz) - p.vx * (p.vy * p.Sy + p.vz * p.Sz)) * cost) /
                (p.vy * p.Sz - p.vz * p.Sy);
  double cos2t = cost * cost - sint * sint;
  double sin2t = (2.0 * sint) * cost;
  double Q = p.Q * cos2t + p.U * sin2t;
  double U = (-p.Q) * sin2t + p.U * cos2t;
  double P2 = (U / p.E) * (U / p.E) + (Q / p.E) * (Q / p.E);
  double sPP2 = sqrt(P / P2);
  p.U = sPP2 * U;
  p.Q = sPP2 * Q;
}

/* ------------------------------------------------------------- temperature */
TP_FN double tp_t4(int i) {
  double d = (double)i;
  double d2 = d * d;
  return d2 * d2;
}
TP_FN double tp_qroot(double x) { return sqrt(sqrt(x)); }

/* the reference's real(i)**4 (Radiation.f:551, 584, 698): single precision,
 * the integer power expanded as (x x)(x x) */
TP_FN float tp_t4f(int i) {
  const float x = (float)i;
  const float x2 = x * x;
  return x2 * x2;
}

/* i^4 + (j^4 - i^4) num / den, the T^4 interpolation of increaseT and
 * determineT, with the powers in double or (single) as the reference forms
 * them: its difference is a single-precision subtraction widened to double */
TP_FN double tp_t4_interp(int i, int j, double num, double den, int single) {
  if (single) {
    const float a = tp_t4f(i), d = tp_t4f(j) - tp_t4f(i);
    return (double)a + ((double)d * num) / den;
  }
  return tp_t4(i) + ((tp_t4(j) - tp_t4(i)) * num) / den;
}

/* determineT, Radiation.f:629-702, on the cell's Planck-mean table kp */
TP_NOINLINE double tp_determine_t(const double *kp, double E1, double Tcur, int single = 0) {
  int iTmin = 1, iTmax = TP_TMAX;
  int iT = (int)(Tcur / 1.0);
  if (iT < 1) iT = 1;
  if (iT > TP_TMAX - 1) iT = TP_TMAX - 1;
  double E = kp[iT];
  double Emax = kp[iTmax];
  double Emin = kp[1];
  if (E1 != E1) return 3.0;
  if (E1 > Emax) return (double)(TP_TMAX - 1);
  if (E1 < Emin) return 1.0;
  int iT0 = iT;
  int niter = 0;
  while ((iTmax - iTmin > 1 || iTmin - iTmax > 1) && niter <= TP_TMAX) {
    niter++;
    iT = (int)(tp_qroot(E1 / E) * (double)iT);
    if (iT == iT0) {
      if (E1 < E) iT = iT0 - 1;
      if (E1 > E) iT = iT0 + 1;
    }
    if (iT <= iTmin) iT = iTmin + 1;
    if (iT >= iTmax) iT = iTmax - 1;
    if (iT <= iTmin) iT = iTmin + 1;
    int c = iT > TP_TMAX ? TP_TMAX : (iT < 1 ? 1 : iT);
    E = kp[c];
    if (E >= E1) {
      iTmax = iT;
      Emax = E;
    }
    if (E <= E1) {
      iTmin = iT;
      Emin = E;
    }
    iT0 = iT;
  }
  if (iTmin == iTmax) return (double)iTmin;
  return tp_qroot(tp_t4_interp(iTmin, iTmax, E1 - Emin, Emax - Emin, single));
}

/* Temperature of a cell with absorbed energy per mass E1: the value the
 * reference's increaseT (upward scan from the cell's current temperature)
 * returns, found by a search over the monotone table: the first i >= 1 with
 * kp[i+1] >= E1 brackets E1 when kp[i] <= E1.  `lo` is a known lower bound
 * of that i (0 when unknown); *ibr returns the bracket (0 when the
 * determineT fallback was taken). */
TP_FN double tp_tinv(const double *kp, double E1, int lo, int *ibr, int single = 0) {
  *ibr = 0;
  if (!(E1 >= kp[1]) || !(E1 <= kp[TP_TMAX])) return tp_determine_t(kp, E1, 0.0, single);
  /* galloping search from lo for the first p in [2, TMAX] with kp[p] >= E1;
   * a hint is used only when kp[lo] < E1 (then lo is below the answer) */
  if (lo < 1 || lo >= TP_TMAX || !(kp[lo] < E1)) lo = 1;
  int a = lo;
  int step = 1, b = a + 1;
  while (b < TP_TMAX && kp[b] < E1) {
    a = b;
    b = a + step;
    step += step;
    if (b > TP_TMAX) b = TP_TMAX;
  }
  /* answer p in (a, b]: first with kp[p] >= E1 */
  int l = a + 1, h = b;
  while (l < h) {
    int mid = (l + h) >> 1;
    if (kp[mid] >= E1)
      h = mid;
    else
      l = mid + 1;
  }
  int i = l - 1;
  *ibr = i;
  double kp0 = kp[i], kp1 = kp[i + 1];
  return tp_qroot(tp_t4_interp(i, i + 1, E1 - kp0, kp1 - kp0, single));
}

/* ------------------------------------------------------------- scattering */
TP_FN void tp_scatangle(const TModel &m, px_stream *r, TPkt &p, const double *F,
                              const double *IF) {
  const double *F11 = F, *F12 = F + 180, *F22 = F + 360, *F33 = F + 540, *F34 = F + 720,
               *F44 = F + 900;
  double IF11 = IF[0] * 180.0, IF12 = IF[1] * 180.0;
  double phi;
  if (p.pol) {
    double Itot = 0.0;
    for (int i = 1; i <= 180; ++i)
      Itot = (Itot + IF11 * p.E) + IF12 * (p.Q * m.cos2phi[i] + p.U * m.sin2phi[i]);
    Itot = tp_rnd(r) * Itot;
    double I1 = 0.0, I0 = 0.0;
    phi = TP_PI;
    for (int i = 1; i <= 180; ++i) {
      I0 = (I0 + IF11 * p.E) + IF12 * (p.Q * m.cos2phi[i] + p.U * m.sin2phi[i]);
      if (I0 > Itot) {
        double wp1 = (I0 - Itot) / (I0 - I1);
        phi = (TP_PI * ((double)i - wp1)) / 180.0;
        break;
      }
      I1 = I0;
    }
  } else {
    phi = tp_rnd(r) * TP_PI;
  }
  double x = p.Sx, y = p.Sy, z = p.Sz;
  tp_rotate(&x, &y, &z, p.vx, p.vy, p.vz, phi);
  if (p.pol) tp_rotate_stokes(p, x, y, z);
  p.Sx = x;
  p.Sy = y;
  p.Sz = z;
  double Fr = 180.0 * (p.E * IF[0] + p.Q * IF[1]);
  Fr = tp_rnd(r) * Fr;
  double Fi = 0.0, FiOld = 0.0, theta = TP_PI;
  int ib = 180;
  for (int i = 1; i <= 180; ++i) {
    Fi = Fi + (TP_PI * m.sinthet[i - 1]) * (F11[i - 1] * p.E + F12[i - 1] * p.Q);
    if (Fi > Fr) {
      theta = (double)i - (Fi - Fr) / (Fi - FiOld);
      theta = (theta * TP_PI) / 180.0;
      ib = i;
      break;
    }
    FiOld = Fi;
  }
  if (tp_rnd(r) < 0.5) theta = -theta;
  int k = ib - 1;
  double E = (0.0 + F11[k] * p.E) + F12[k] * p.Q;
  double Q = (0.0 + F12[k] * p.E) + F22[k] * p.Q;
  double U = 0.0 + F33[k] * p.U;
  double Fs = (theta >= 0.0 && !signbit(theta)) ? fabs(F34[k]) : -fabs(F34[k]);
  U = U + Fs * p.V;
  double V = (0.0 - Fs * p.U) + F44[k] * p.V;
  if (E != 0.0) {
    p.Q = (p.E * Q) / E;
    p.U = (p.E * U) / E;
    p.V = (p.E * V) / E;
  }
  tp_rotate(&p.vx, &p.vy, &p.vz, p.Sx, p.Sy, p.Sz, theta);
  double rr = sqrt((p.vx * p.vx + p.vy * p.vy) + p.vz * p.vz);
  p.vx /= rr;
  p.vy /= rr;
  p.vz /= rr;
  rr = sqrt((p.Sx * p.Sx + p.Sy * p.Sy) + p.Sz * p.Sz);
  p.Sx /= rr;
  p.Sy /= rr;
  p.Sz /= rr;
  if (ib != 1 && ib != 180) p.pol = 1;
}

/* ------------------------------------------------------------- interaction */
TP_FN void tp_interact(const TModel &m, const TAcc &A, px_stream *r, TPkt &p, TLocal &L) {
  const int c = p.i * m.nc + (p.j - 1);
  const int nlam = m.nlam;
  const double *KabsT = m.KabsTot + (size_t)c * nlam;
  const double *KscaT = m.KscaTot + (size_t)c * nlam;
  double Ksca = KscaT[p.ilam1] * p.wl1 + KscaT[p.ilam2] * p.wl2;
  double Kext = Ksca + (KabsT[p.ilam1] * p.wl1 + KabsT[p.ilam2] * p.wl2);
  double KabsTot = Kext - Ksca;
  double Albedo = Ksca / Kext;
  L.cnt[TC_INTERACT]++;
  if (!m.scattering || tp_rnd(r) > Albedo) {
    L.cnt[TC_ABSORB]++;
    if (A.Nabs) tp_addi(&A.Nabs[c], 1);
    p.scatt = 0;
    p.pol = 0;
    p.Q = 0.0;
    p.U = 0.0;
    p.V = 0.0;
    const double *kp = m.KpCell + (m.uniform_mix ? (size_t)0 : (size_t)c * TP_TT);
    const double dE = (p.E * (KabsTot - 0.0)) / KabsTot;
    const double Eold = tp_add(&A.Eabs[c], dE);
    const double Enew = Eold + dE;
    const double mass = m.mass[c];
    int ib0, ib1;
    const double T0 = tp_tinv(kp, Eold / mass, 0, &ib0, m.t4single);
    const double T1 = tp_tinv(kp, Enew / mass, ib0, &ib1, m.t4single);
    int iT0 = (int)(T0 / 1.0), iT1 = (int)(T1 / 1.0);
    double epsT0 = T0 - (double)iT0 * 1.0, epsT1 = T1 - (double)iT1 * 1.0;
    if (iT0 >= TP_TMAX - 1) iT0 = TP_TMAX - 2;
    if (iT1 >= TP_TMAX - 1) iT1 = TP_TMAX - 1;
    if (iT0 < 1) iT0 = 1;
    if (iT1 < 2) iT1 = 2;
    tp_emit_dir(r, p, L);
    if (iT0 == iT1 && m.uniform_mix) {
      /* cumulative table of (BB(iT0+1)-BB(iT0))*KabsTot, built in the scan order */
      double kpe = kp[iT0 + 1] - kp[iT0];
      if (kpe == 0.0) {
        /* the reference zeroes the spectrum: the scan stops at the first
         * (empty) interval with weight 1 */
        (void)tp_rnd(r);
        p.wl1 = 1.0;
        p.wl2 = 0.0;
        p.ilam1 = 0;
        p.ilam2 = 1;
      } else {
        tp_pick_cdf(m, p, m.emit_cdf + (size_t)iT0 * (nlam - 1), tp_rnd(r) * kpe);
      }
    } else {
      double kpe;
      if (iT0 == iT1)
        kpe = kp[iT0 + 1] - kp[iT0];
      else
        kpe = ((epsT1 * kp[iT1 + 1] + (1.0 - epsT1) * kp[iT1]) - epsT0 * kp[iT0 + 1]) - (1.0 - epsT0) * kp[iT0];
      const bool zero = kpe == 0.0;
      if (zero) kpe = 0.0 / KabsTot;
      double Lr = tp_rnd(r) * kpe;
      /* linear scan of the re-emission spectrum (Radiation.f:187-213, :966-988) */
      const double *BB = m.BB;
      double Ltold = 0.0, Lt = 0.0, sprev;
      bool found = false;
      {
        const double *B = BB + 0 * (size_t)TP_TT;
        if (zero)
          sprev = 0.0;
        else if (iT0 == iT1)
          sprev = (B[iT0 + 1] - B[iT0]) * KabsT[0];
        else
          sprev = (((epsT1 * B[iT1 + 1] + (1.0 - epsT1) * B[iT1]) - epsT0 * B[iT0 + 1]) - (1.0 - epsT0) * B[iT0]) * KabsT[0];
      }
      for (int i = 0; i < nlam - 1; ++i) {
        const double *B = BB + (size_t)(i + 1) * TP_TT;
        double snext;
        if (zero)
          snext = 0.0;
        else if (iT0 == iT1)
          snext = (B[iT0 + 1] - B[iT0]) * KabsT[i + 1];
        else
          snext = (((epsT1 * B[iT1 + 1] + (1.0 - epsT1) * B[iT1]) - epsT0 * B[iT0 + 1]) - (1.0 - epsT0) * B[iT0]) * KabsT[i + 1];
        Lt = Lt + m.dnu_half[i] * (sprev + snext);
        if (Lt >= Lr) {
          double d = Lt - Ltold;
          p.wl1 = d != 0.0 ? (Lr - Ltold) / d : 1.0;
          p.wl2 = 1.0 - p.wl1;
          p.ilam1 = i;
          p.ilam2 = i + 1;
          found = true;
          break;
        }
        Ltold = Lt;
        sprev = snext;
      }
      if (!found) {
        p.wl1 = 0.0;
        p.wl2 = 1.0;
        p.ilam1 = nlam - 2;
        p.ilam2 = nlam - 1;
      }
    }
    A.T[c] = T1;
  } else {
    L.cnt[TC_SCATTER]++;
    p.scatt = 1;
    if (m.scat_how == 1) {
      tp_randomdirection(r, &p.vx, &p.vy, &p.vz);
    } else {
      double KscaR = Ksca * tp_rnd(r);
      const double *F = nullptr, *IF = nullptr;
      const double *w = m.comp_w + (size_t)c * m.ncomp;
      int qlast = -1, llast = p.ilam1;
      for (int q = 0; q < m.ncomp; ++q) {
        double w1 = w[q];
        double w2 = (w1 * p.wl2) * m.Ksca_c[(size_t)q * nlam + p.ilam2];
        KscaR = KscaR - w2;
        if (KscaR < 0.0) {
          F = m.F_c + ((size_t)q * nlam + p.ilam2) * 1080;
          IF = m.IF_c + ((size_t)q * nlam + p.ilam2) * 2;
          break;
        }
        w1 = (w1 * p.wl1) * m.Ksca_c[(size_t)q * nlam + p.ilam1];
        KscaR = KscaR - w1;
        if (KscaR < 0.0) {
          F = m.F_c + ((size_t)q * nlam + p.ilam1) * 1080;
          IF = m.IF_c + ((size_t)q * nlam + p.ilam1) * 2;
          break;
        }
        if (w2 > 0.0) { qlast = q; llast = p.ilam2; }
        if (w1 > 0.0) { qlast = q; llast = p.ilam1; }
      }
      if (F == nullptr) {
        /* rounding left KscaR >= 0: the reference averages the matrices
         * (Radiation.f:293-315); the device takes the last component with
         * weight (counted) */
        L.cnt[TC_AVGMAT]++;
        if (qlast < 0) qlast = 0;
        F = m.F_c + ((size_t)qlast * nlam + llast) * 1080;
        IF = m.IF_c + ((size_t)qlast * nlam + llast) * 2;
      }
      tp_scatangle(m, r, p, F, IF);
    }
  }
}

/* ------------------------------------------------------------- random walk */
TP_FN double tp_mindist(const TModel &m, const TPkt &p) {
  double rho = p.x * p.x + p.y * p.y;
  double r = sqrt(rho + p.z * p.z);
  rho = sqrt(rho);
  double z = fabs(p.z);
  double R1 = m.R[p.i], R2 = m.R[p.i + 1];
  double T1 = m.Theta[p.j - 1], T2 = m.Theta[p.j];
  double ST1 = m.SinTheta[p.j - 1], ST2 = m.SinTheta[p.j];
  double vR1 = fabs(r - R1), vR2 = fabs(R2 - r);
  double vT1 = fabs(T1 * rho - ST1 * z), vT2 = fabs(T2 * rho - ST2 * z);
  double d = vR1;
  if (vR2 < d) d = vR2;
  if (vT1 < d) d = vT1;
  if (vT2 < d) d = vT2;
  return d;
}

/* Numerical Recipes hunt (Subroutines.f:2086-2132), 1-based jlo in/out */
TP_FN void tp_hunt(const double *xx, int n, double x, int *jlo) {
  int jhi, jm, inc;
  const bool ascnd = xx[n - 1] >= xx[0];
  if (*jlo <= 0 || *jlo > n) {
    *jlo = 0;
    jhi = n + 1;
  } else {
    inc = 1;
    if ((x >= xx[*jlo - 1]) == ascnd) {
      for (;;) {
        jhi = *jlo + inc;
        if (jhi > n) {
          jhi = n + 1;
          break;
        } else if ((x >= xx[jhi - 1]) == ascnd) {
          *jlo = jhi;
          inc += inc;
        } else {
          break;
        }
      }
    } else {
      jhi = *jlo;
      for (;;) {
        *jlo = jhi - inc;
        if (*jlo < 1) {
          *jlo = 0;
          break;
        } else if ((x < xx[*jlo - 1]) == ascnd) {
          jhi = *jlo;
          inc += inc;
        } else {
          break;
        }
      }
    }
  }
  while (jhi - *jlo != 1) {
    jm = (jhi + *jlo) / 2;
    if ((x >= xx[jm - 1]) == ascnd)
      *jlo = jm;
    else
      jhi = jm;
  }
  if (x == xx[n - 1]) *jlo = n - 1;
  if (x == xx[0]) *jlo = 1;
}

TP_FN int tp_random_walk(const TModel &m, const TAcc &A, px_stream *r, TPkt &p, double dmin,
                               TLocal &L) {
  const int c = p.i * m.nc + (p.j - 1);
  int iT = (int)(A.T[c] / 1.0);
  if (iT == 0) iT = 1;
  if (iT > TP_TMAX) iT = TP_TMAX;
  if (iT > TP_TMAX - 1) iT = TP_TMAX - 1;
  const int row = m.kd_index[c];
  if (row < 0) return 0;
  const double Kext = m.KDext[(size_t)row * TP_TT + iT];
  const double lr = 1.0 / ((TP_AU * Kext) * m.dens[c]);
  if (dmin <= m.factRW * lr) return 0;
  double x = tp_rnd(r);
  int iy = 1;
  tp_hunt(m.rw_phi, TP_NY, x, &iy);
  double v = (((-3.0 * dm_log(m.rw_y[iy - 1])) * (dmin * dmin)) / (lr * (TP_PI * TP_PI)));
  const double Kabs = m.KDabs[(size_t)row * TP_TT + iT];
  tp_randomdirection(r, &p.vx, &p.vy, &p.vz);
  p.x = p.x + dmin * p.vx;
  p.y = p.y + dmin * p.vy;
  p.z = p.z + dmin * p.vz;
  const double EJv = (p.E * v) * TP_AU;
  const double dEa = (EJv * Kabs) * m.dens[c];
  const double Eold = tp_add(&A.Eabs[c], dEa);
  tp_add(&A.EJv[c], EJv * Kabs);
  p.nEJv = p.nEJv + EJv * Kabs;
  const double *kp = m.KpCell + (m.uniform_mix ? (size_t)0 : (size_t)c * TP_TT);
  int ib;
  A.T[c] = tp_tinv(kp, (Eold + dEa) / m.mass[c], 0, &ib, m.t4single);
  L.tautot += v / dmin;
  L.cnt[TC_RWSTEP]++;
  return 1;
}

/* ------------------------------------------------------------- trace2d */
/* returns 0 interaction, 1 escape, 2 star hit / abandoned, -1 geometry
 * failure */
TP_FN int tp_trace2d(const TModel &m, const TAcc &A, px_stream *r, TPkt &p, double tau0,
                           TLocal &L) {
  const int nlam = m.nlam;
  double tau = 0.0;
  int ntrace = 0;
  if (m.rw && m.thick[p.i * m.nc + (p.j - 1)] && !p.onEdge) {
    for (;;) {
      double dmin = tp_mindist(m, p);
      if (!tp_random_walk(m, A, r, p, dmin, L)) break;
      double vx, vy, vz, inp;
      do {
        tp_randomdirection(r, &vx, &vy, &vz);
        inp = (p.vx * vx + p.vy * vy) + p.vz * vz;
      } while (inp < 0.0);
      p.vx = vx;
      p.vy = vy;
      p.vz = vz;
    }
  }
  for (;;) {
    const int c = p.i * m.nc + (p.j - 1);
    if (tp_exch(&A.lastphot[c], p.pid1) != p.pid1) tp_addi(&A.Ni[c], 1);
    const double *KabsT = m.KabsTot + (size_t)c * nlam;
    double Kabs = KabsT[p.ilam1] * p.wl1 + KabsT[p.ilam2] * p.wl2;
    double Kext = Kabs;
    if (m.scattering) {
      const double *KscaT = m.KscaTot + (size_t)c * nlam;
      Kext = (KscaT[p.ilam1] * p.wl1 + KscaT[p.ilam2] * p.wl2) + Kabs;
    }
    double v;
    int inext, jnext;
    if (tp_trace2edge(m, p, &v, &inext, &jnext)) return -1;
    L.cnt[TC_CROSS]++;
    double tau1 = ((Kext * v) * m.dens[c]) * TP_AU;
    if (tau + tau1 > tau0) {
      v = (v * (tau0 - tau)) / tau1;
      tau1 = tau0 - tau;
      L.tautot += tau1;
      p.x = p.x + p.vx * v;
      p.y = p.y + p.vy * v;
      p.z = p.z + p.vz * v;
      p.onEdge = 0;
      double EJv = (p.E * v) * TP_AU;
      tp_add(&A.EJv[c], EJv * Kabs);
      p.nEJv = p.nEJv + EJv * Kabs;
      return 0;
    }
    p.x = p.x + p.vx * v;
    p.y = p.y + p.vy * v;
    p.z = p.z + p.vz * v;
    double EJv = (p.E * v) * TP_AU;
    p.nEJv = p.nEJv + EJv * Kabs;
    tp_add(&A.EJv2[c], p.nEJv * p.nEJv);
    p.nEJv = 0.0;
    tp_add(&A.EJv[c], EJv * Kabs);
    p.onEdge = 1;
    tau = tau + tau1;
    L.tautot += tau1;
    if (inext >= m.nr) return 1;
    if (inext < 0) return 2;
    p.i = inext;
    p.j = jnext;
    ntrace++;
    if (tau < 0.0) return 2;
    if (ntrace > m.nr * m.nt * 2) {
      L.cnt[TC_ABANDON]++;
      return 2;
    }
  }
}

/* ------------------------------------------------------------- one packet */
TP_FN void tp_run_packet(const TModel &m, const TAcc &A0, int64_t pid, TLocal &L) {
  const TAcc A = tp_run_acc(A0, pid);
  px_stream rs;
  px_init(&rs, m.seed, (uint64_t)pid);
  px_stream *r = &rs;
  TPkt p;
  p.pid1 = (int)(pid + 1);
  p.Q = p.U = p.V = 0.0;
  p.pol = 0;
  p.scatt = 0;
  for (;;) {
    /* (re-)emission from the star */
    p.nEJv = 0.0;
    (void)tp_rnd(r); /* where_emit */
    double x, y, z;
    tp_randomdirection(r, &x, &y, &z);
    p.x = m.R0 * x;
    p.y = m.R0 * y;
    p.z = m.R0 * z;
    tp_emit_dir(r, p, L);
    tp_pick_cdf(m, p, m.star_cdf, tp_rnd(r) * m.Lstar);
    p.E = m.Epkt;
    tp_randomdirection(r, &p.vx, &p.vy, &p.vz);
    if ((p.x * p.vx + p.y * p.vy) + p.z * p.vz < 0.0) {
      p.vx = -p.vx;
      p.vy = -p.vy;
      p.vz = -p.vz;
    }
    p.edgeNr = 1;
    p.onEdge = 1;
    const double ct = fabs(p.z) / m.R0;
    p.i = 0;
    p.j = -1;
    for (int j = 1; j <= m.nt - 1; ++j)
      if (ct < m.Theta[j - 1] && ct > m.Theta[j]) p.j = j;
    if (p.j < 0) {
      for (int j = 1; j <= m.nt - 1; ++j)
        if (ct >= m.Theta[j]) {
          p.j = j;
          break;
        }
      if (p.j < 0) p.j = m.nt - 1;
    }
    if (m.scattering) {
      p.pol = 0;
      p.scatt = 0;
      p.Q = p.U = p.V = 0.0;
      tp_set_s(p);
    }
    double tau = -dm_log(tp_rnd(r));
    for (;;) {
      int st = tp_trace2d(m, A, r, p, tau, L);
      if (st < 0) {
        L.cnt[TC_GEOFAIL]++;
        return;
      }
      if (st == 2) {
        L.cnt[TC_HITSTAR]++;
        break; /* re-launch from the star */
      }
      if (st == 1) {
        L.cnt[TC_ESCAPE]++;
        double av = p.vz > 0.0 ? p.vz : -p.vz;
        int ia = (int)(av * (double)TP_NANG + 1.0);
        if (ia > TP_NANG) ia = TP_NANG;
        int il = (p.wl1 > p.wl2) ? p.ilam1 : p.ilam2;
        size_t k = (size_t)il * (TP_NANG + 1) + ia;
        double wangle = 1.0 / ((double)ia / (double)TP_NANG - (double)(ia - 1) / (double)TP_NANG);
        double add = ((wangle * p.E) * m.wlam[il]) / m.nruns_d;
        tp_add(&A.spec[k], add);
        tp_addi(&A.ispec[k], 1);
        if (p.scatt) tp_add(&A.scatspec[k], add);
        return;
      }
      tp_interact(m, A, r, p, L);
      if (m.maxinteract > 0) {
        if (tp_rnd(r) < 1.0 / (double)m.maxinteract) {
          L.cnt[TC_OVERFLOW]++;
          return;
        }
        p.E = (p.E * (double)m.maxinteract) / (double)(m.maxinteract - 1);
      }
      tau = -dm_log(tp_rnd(r));
    }
  }
}

#endif /* MCMAX_TRANSPORT_CORE_CUH */
