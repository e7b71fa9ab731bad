/*
 * transport_fast.cuh -- the MCMax packet loop restructured for the GPU,
 * templated on the precision of the direction / Stokes / optical-depth /
 * opacity arithmetic (R = double: "fp64", R = float: "mixed").  Positions,
 * the sphere/cone intersection quadratics, packet energies, the per-cell
 * energy accumulators and the Bjorkman-Wood temperature inversion are FP64 in
 * both forms.
 *
 * Same physics and the same random-number consumption as the reference-order
 * kernel (transport_core.cuh), with the per-event latency cut:
 *   - geometry edges, the star spectrum CDF, the opacity rows of a uniform
 *     mixture, component scattering opacities and the cumulative phi tables
 *     live in shared memory;
 *   - the opacity at the packet's wavelength is formed once per emission or
 *     scattering-wavelength change (uniform mixture), not once per crossing;
 *   - wavelength re-emission (Radiation.f:187-213, :966-988) samples from
 *     cumulative tables by binary search: C(iT)[i] = cumulative of BB(iT) K
 *     and D(iT)[i] = cumulative of (BB(iT+1) - BB(iT)) K, so the spectrum of
 *     a (T0 -> T1) jump has the cumulative [C(iT1) + e1 D(iT1)] -
 *     [C(iT0) + e0 D(iT0)] (exactly the reference's interpolated Delta-B);
 *   - the scattering angle (Radiation.f:434-452) samples from the
 *     cumulative A_k = sum pi sin(th_i) F11_i, B_k = sum pi sin(th_i) F12_i
 *     with F_k = E A_k + Q B_k, and the polarised azimuth (:393-420) from
 *     cumulative sums of cos 2phi / sin 2phi, both by binary search;
 *   - the temperature inversion gallops from a per-cell bracket hint (the
 *     absorbed energy of a cell only grows, so any stored bracket is a valid
 *     lower bound).
 * Stokes parameters are carried as fractions of E (q = Q/E ...), which is
 * what the reference's renormalisation (Radiation.f:480-483) keeps invariant.
 * Results agree with the reference-order kernel up to floating-point
 * reassociation; the checks are statistical against the CPU oracle and
 * paired (identical Philox streams) against the reference-order kernel.
 */
#ifndef MCMAX_TRANSPORT_FAST_CUH
#define MCMAX_TRANSPORT_FAST_CUH

#include "transport_core.cuh"

template <class R>
struct FModel {
  int nr, nt, nc, ncell, nlam, ncomp;
  int scattering, scat_how, uniform_mix, rw, pol_tables;
  double factRW, R0, Lstar, Epkt, nruns_d;
  int64_t nphot, maxinteract, pid0;
  uint64_t seed;
  /* shared-memory copies (or global when not uniform) */
  const double *Rr, *Theta, *SinTheta, *star_cdf;
  const R *KabsRow, *KextRow;  /* uniform mixture: one row each */
  const R *Ksca_c;             /* ncomp*nlam */
  const double *c2cum, *s2cum; /* 181: cumulative cos/sin(2 phi_i), i = 1..k */
  /* global */
  const double *dens, *mass, *wlam;
  const R *KabsTotR, *KextTotR; /* ncell*nlam (non-uniform mixtures) */
  const double *KabsTot;        /* ncell*nlam, for the per-cell scan */
  const double *BB, *dnu_half;
  const double *BBT;            /* non-uniform mixtures: BB temperature-major */
  const double *KpCell;         /* uniform: 1 row, else ncell rows */
  const double *Ccum, *Dcum;    /* uniform mixture: TT*(nlam-1) */
  const double *comp_w;
  const R *scatA, *scatB;       /* ncomp*nlam*180 */
  const unsigned char *scatG;   /* ncomp*nlam*NGUIDE: first bin with A > k/NGUIDE of the total */
  const unsigned short *emitG;  /* TMAX*NGUIDE: same for the rows of Dcum */
  const R *F6;                  /* ncomp*nlam*1080 */
  const double *IF_c;
  const double *KDext, *KDabs, *rw_logy, *rw_phi;
  const int *kd_index;
  const unsigned char *thick;
  const double *rw_dmin;        /* factRW x the cell's shortest mean free path */
  double maxruntime;            /* seconds; > 0: MCRadiation.f:323-342 */
  int t4single;                 /* 1: single-precision i^4 in the temperature inversion */
};

#define F_NGUIDE 32

/* member functions of the table functors (TP_FN is `static` on the host) */
#if defined(__CUDACC__)
#define F_MFN __host__ __device__ __forceinline__
#else
#define F_MFN inline
#endif

/* cold paths (interactions, random walk, emission) can be compiled out of
 * line to keep the crossing loop small in the instruction cache */
#if defined(__CUDACC__) && defined(F_COLD_NOINLINE)
#define F_COLD __host__ __device__ __noinline__
#else
#define F_COLD TP_FN
#endif

/* first index i in [0,n) with f(i) > v (or >= when ge), starting from a
 * guess and walking; f is non-decreasing */
template <class F>
TP_FN int f_walk(F f, int n, int i, double v, bool ge) {
  if (i < 0) i = 0;
  if (i > n) i = n;
  auto above = [&](int k) { return ge ? f(k) >= v : f(k) > v; };
  if (i < n && above(i)) {
    while (i > 0 && above(i - 1)) --i;
  } else {
    while (i < n && !above(i)) ++i;
  }
  return i;
}

template <class R>
struct FPkt {
  double x, y, z, E, nEJv;
  /* transport direction: FP64 and re-normalised after every FP32 rotation,
   * so the FP64 intersection quadratics (which assume |v| = 1) put the packet
   * on the cell faces */
  double vx, vy, vz;
  R q, u, v;    /* Stokes / E */
  R Sx, Sy, Sz;
  R wl1, wl2;
  R kabs, kext; /* at the packet wavelength, uniform mixture */
  R kabs_i, ksca_i; /* at the interaction point (set when a trace ends inside a cell) */
  int ilam1, i, j, edgeNr, onEdge, scatt, pol, pid1;
  int cprev1, cprev2; /* last two cells this packet entered */
};

template <class R>
struct FOps;
template <>
struct FOps<double> {
  TP_SFN double sqrt_(double x) { return sqrt(x); }
  TP_SFN double log_(double x) { return log(x); }
  TP_SFN void sincos_(double x, double *s, double *c) { sincos(x, s, c); }
  TP_SFN double u(double x) { return x; }
};
template <>
struct FOps<float> {
  TP_SFN float sqrt_(float x) { return sqrtf(x); }
  TP_SFN float log_(float x) { return logf(x); }
  TP_SFN void sincos_(float x, float *s, float *c) { sincosf(x, s, c); }
  /* a draw in (0,1) as float, kept < 1 */
  TP_SFN float u(double x) {
    float f = (float)x;
    return f < 1.0f ? f : 0.99999994f;
  }
};

template <class R>
TP_FN void f_randomdirection(px_stream *r, R *x, R *y, R *z) {
  typedef FOps<R> O;
  R rr;
  for (;;) {
    *x = (R)2 * O::u(px_next(r)) - (R)1;
    *y = (R)2 * O::u(px_next(r)) - (R)1;
    *z = (R)2 * O::u(px_next(r)) - (R)1;
    rr = (*x) * (*x) + (*y) * (*y) + (*z) * (*z);
    if (!(rr > (R)1)) break;
  }
  rr = (R)1 / O::sqrt_(rr);
  *x *= rr;
  *y *= rr;
  *z *= rr;
}

template <class R>
TP_FN void f_set_dir(FPkt<R> &p, R x, R y, R z) {
  const double dx = (double)x, dy = (double)y, dz = (double)z;
  const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
  p.vx = dx * inv;
  p.vy = dy * inv;
  p.vz = dz * inv;
}

template <class R>
TP_FN void f_set_s(FPkt<R> &p) {
  typedef FOps<R> O;
  R x = (R)-p.vy, y = (R)p.vx;
  R r = (R)1 / O::sqrt_(x * x + y * y);
  p.Sx = x * r;
  p.Sy = y * r;
  p.Sz = (R)0;
}

/* first index in [0,n) with cdf[i] >= v (n when none) */
TP_FN int f_lower_bound(const double *cdf, int n, double v) {
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

template <class R>
TP_FN void f_set_lambda(const FModel<R> &m, FPkt<R> &p) {
  if (m.uniform_mix) {
    const int l = p.ilam1;
    p.kabs = m.KabsRow[l] * p.wl1 + m.KabsRow[l + 1] * p.wl2;
    p.kext = m.KextRow[l] * p.wl1 + m.KextRow[l + 1] * p.wl2;
  }
}

/* interval pick on a cumulative table (shared by star and re-emission) */
template <class R>
TP_FN void f_pick(const FModel<R> &m, FPkt<R> &p, int i, double Lt, double Ltold, double Lr) {
  const int n = m.nlam - 1;
  if (i < n) {
    double d = Lt - Ltold;
    double w = d != 0.0 ? (Lr - Ltold) / d : 1.0;
    p.wl1 = (R)w;
    p.wl2 = (R)(1.0 - w);
    p.ilam1 = i;
  } else {
    p.wl1 = (R)0;
    p.wl2 = (R)1;
    p.ilam1 = m.nlam - 2;
  }
}

/* ------------------------------------------------------------- geometry */
/* Distance to the next cell boundary (Trace2edge, MCRadiation.f:1150-1272),
 * same values as tp_trace2edge.  tp_trace2edge evaluates only the
 * intersections each entry edge needs, in five branches; lanes of a warp
 * that entered their cells through different edges then run those branches
 * one after the other.  Here the two sphere and two cone intersections are
 * evaluated once for every lane and the entry-edge rules (skip the sphere or
 * cone just crossed, the re-hit of the same sphere, the midplane plane, the
 * same-cone re-hit) replace values afterwards.  The fall-back of the
 * reference (nothing hit: evaluate all four plainly) is the plain values. */
template <class R>
TP_FN int f_trace2edge(const FModel<R> &m, FPkt<R> &p, double *v, int *inext, int *jnext) {
  const int nt = m.nt;
  TPkt t;
  t.z = p.z;
  t.vz = p.vz;
  const double r = (p.x * p.x + p.y * p.y) + p.z * p.z;
  const double Ra = m.Rr[p.i], Rb = m.Rr[p.i + 1];
  const double Ta = m.Theta[p.j - 1], Tb = m.Theta[p.j];
  const double R1 = Ra * Ra, R2 = Rb * Rb, T1 = Ta * Ta, T2 = Tb * Tb;
  const double b = 2.0 * ((p.x * p.vx + p.y * p.vy) + p.z * p.vz);
  double pvR1, pvR2, pvT1, pvT2;
  const int phR1 = tp_hitR(R1, r, b, &pvR1);
  const int phR2 = tp_hitR(R2, r, b, &pvR2);
  const int phT1 = tp_hitT(t, T1, r, b, &pvT1);
  const int phT2 = tp_hitT(t, T2, r, b, &pvT2);
  int hR1 = phR1, hR2 = phR2, hT1 = phT1, hT2 = phT2;
  double vR1 = pvR1, vR2 = pvR2, vT1 = pvT1, vT2 = pvT2;
  if (p.onEdge) {
    const int e = p.edgeNr;
    if (e == 1) {
      hR1 = 0;
      vR1 = 1e200;
    } else if (e == 2) {
      hR2 = 1;
      vR2 = -b;
    } else if (e == 3) {
      hT1 = 0;
      vT1 = 1e200;
      if (p.j == nt - 1) {
        vT2 = -p.z / p.vz;
        hT2 = vT2 > 0.0;
      }
    } else {
      if (p.j == 1) {
        hT1 = 0;
        vT1 = 1e200;
      }
      if (p.j != nt - 1) {
        hT2 = tp_hitTsame(t, T2, b, &vT2);
      } else {
        hT2 = 0;
        vT2 = 1e200;
      }
    }
  }
  if (!hR1 && !hR2 && !hT1 && !hT2) {
    hR1 = phR1; hR2 = phR2; hT1 = phT1; hT2 = phT2;
    vR1 = pvR1; vR2 = pvR2; vT1 = pvT1; vT2 = pvT2;
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

/* ------------------------------------------------------------- rotations */
template <class R>
TP_FN void f_rotate(R *x, R *y, R *z, R u, R v, R w, R theta) {
  R sint, cost;
  FOps<R>::sincos_(theta, &sint, &cost);
  R u2 = u * u, v2 = v * v, w2 = w * w;
  R inp = *x * u + *y * v + *z * w;
  R y1 = u * inp + (*x * (v2 + w2) - u * (v * *y + w * *z)) * cost + (v * *z - w * *y) * sint;
  R y2 = v * inp + (*y * (u2 + w2) - v * (u * *x + w * *z)) * cost + (w * *x - u * *z) * sint;
  R y3 = w * inp + (*z * (u2 + v2) - w * (u * *x + v * *y)) * cost + (u * *y - v * *x) * sint;
  *x = y1;
  *y = y2;
  *z = y3;
}

template <class R>
TP_FN void f_rotate_stokes(FPkt<R> &p, R x, R y, R z) {
  typedef FOps<R> O;
  R P = p.u * p.u + p.q * p.q;
  if (P == (R)0) return;
  const R vx = (R)p.vx, vy = (R)p.vy, vz = (R)p.vz;
  R cost = p.Sx * x + p.Sy * y + p.Sz * z;
  R sint = (x - (p.Sx * (vy * vy + vz * vz) - vx * (vy * p.Sy + vz * p.Sz)) * cost) / (vy * p.Sz - vz * p.Sy);
  R cos2t = cost * cost - sint * sint;
  R sin2t = (R)2 * sint * cost;
  R Q = p.q * cos2t + p.u * sin2t;
  R U = -p.q * sin2t + p.u * cos2t;
  R P2 = U * U + Q * Q;
  R s = O::sqrt_(P / P2);
  p.u = s * U;
  p.q = s * Q;
}

/* ------------------------------------------------------------- scattering */
template <class R>
TP_FN void f_scatangle(const FModel<R> &m, px_stream *r, FPkt<R> &p, int mat) {
  typedef FOps<R> O;
  const R *A = m.scatA + (size_t)mat * 180;
  const R *B = m.scatB + (size_t)mat * 180;
  const R *F = m.F6 + (size_t)mat * 1080;
  R phi;
  if (p.pol) {
    /* I0(k) = k IF11 + IF12 (q C_k + u S_k), IF scaled by 180 as the
     * reference does; monotone in k because |F12| <= F11 */
    const double if11 = m.IF_c[2 * mat] * 180.0, if12 = m.IF_c[2 * mat + 1] * 180.0;
    const double qd = (double)p.q, ud = (double)p.u;
    const double Itot = 180.0 * if11 + if12 * (qd * m.c2cum[180] + ud * m.s2cum[180]);
    const double It = px_next(r) * Itot;
    int lo = 1, hi = 181; /* first k in [1,180] with I0(k) > It; 181 = none */
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      double I0 = (double)mid * if11 + if12 * (qd * m.c2cum[mid] + ud * m.s2cum[mid]);
      if (I0 > It)
        hi = mid;
      else
        lo = mid + 1;
    }
    if (lo <= 180) {
      double I0 = (double)lo * if11 + if12 * (qd * m.c2cum[lo] + ud * m.s2cum[lo]);
      double I1 = (double)(lo - 1) * if11 + if12 * (qd * m.c2cum[lo - 1] + ud * m.s2cum[lo - 1]);
      double wp1 = (I0 - It) / (I0 - I1);
      phi = (R)(TP_PI * ((double)lo - wp1) / 180.0);
    } else {
      phi = (R)TP_PI;
    }
  } else {
    phi = O::u(px_next(r)) * (R)TP_PI;
  }
  R x = p.Sx, y = p.Sy, z = p.Sz;
  f_rotate<R>(&x, &y, &z, (R)p.vx, (R)p.vy, (R)p.vz, phi);
  if (p.pol) f_rotate_stokes<R>(p, x, y, z);
  p.Sx = x;
  p.Sy = y;
  p.Sz = z;
  /* scattering angle: F(k) = A_k + q B_k (per unit E); the guide table of
   * A (q = 0) gives the starting bin, a short walk corrects for q */
  const R q = p.q;
  const R Ftot = A[179] + q * B[179];
  const R xr = O::u(px_next(r));
  const R Fr = xr * Ftot;
  int gk = (int)(xr * (R)F_NGUIDE);
  if (gk > F_NGUIDE - 1) gk = F_NGUIDE - 1;
  const int lo = f_walk([&](int k) { return (double)(A[k] + q * B[k]); }, 180,
                        (int)m.scatG[(size_t)mat * F_NGUIDE + gk], (double)Fr, false);
  R theta;
  int ib;
  if (lo < 180) {
    R Fi = A[lo] + q * B[lo];
    R Fo = lo > 0 ? A[lo - 1] + q * B[lo - 1] : (R)0;
    theta = ((R)(lo + 1) - (Fi - Fr) / (Fi - Fo)) * (R)(TP_PI / 180.0);
    ib = lo + 1;
  } else {
    theta = (R)TP_PI;
    ib = 180;
  }
  if (px_next(r) < 0.5) theta = -theta;
  const int k = ib - 1;
  const R F11 = F[k], F12 = F[180 + k], F22 = F[360 + k], F33 = F[540 + k], F34 = F[720 + k], F44 = F[900 + k];
  const R E = F11 + F12 * p.q;
  const R Q = F12 + F22 * p.q;
  R U = F33 * p.u;
  const R Fs = theta >= (R)0 ? (F34 >= (R)0 ? F34 : -F34) : (F34 >= (R)0 ? -F34 : F34);
  U = U + Fs * p.v;
  const R V = -Fs * p.u + F44 * p.v;
  if (E != (R)0) {
    const R ie = (R)1 / E;
    p.q = Q * ie;
    p.u = U * ie;
    p.v = V * ie;
  }
  R vx = (R)p.vx, vy = (R)p.vy, vz = (R)p.vz;
  f_rotate<R>(&vx, &vy, &vz, p.Sx, p.Sy, p.Sz, theta);
  f_set_dir<R>(p, vx, vy, vz);
  R rr = (R)1 / O::sqrt_(p.Sx * p.Sx + p.Sy * p.Sy + p.Sz * p.Sz);
  p.Sx *= rr;
  p.Sy *= rr;
  p.Sz *= rr;
  if (ib != 1 && ib != 180) p.pol = 1;
}

/* ------------------------------------------------------------- temperature */
/* gallop from `lo` (a valid lower bound of the bracket) */
TP_FN double f_tinv(const double *kp, double E1, int lo, int *ibr, int single) {
  return tp_tinv(kp, E1, lo, ibr, single);
}

/* ------------------------------------------------------------- event steps
 * The packet's life as a sequence of events.  One event advances one packet
 * by one step of the reference's loop and consumes the same random numbers
 * in the same order, so a packet is the same packet whether its events run
 * back to back (f_run_packet: the host replay and the batched kernel) or
 * interleaved with other packets' events by the warp scheduler of the
 * single-model kernel.
 *
 *   FS_EMIT     star emission (MCRadiation.f:353-382) and the first tau
 *   FS_RW       one modified-random-walk jump, or none (RandomWalk.f:47-147)
 *   FS_TRACE    one cell crossing of trace2d (MCRadiation.f:941-1138)
 *   FS_ABSORB   absorption + Bjorkman-Wood re-emission (Radiation.f:41-258)
 *   FS_SCATTER  scattering (Radiation.f:259-355, 381-495)
 * An interaction ends with the overflow roulette and the next tau
 * (MCRadiation.f:554-573); a crossing can end the packet (escape: SED bin,
 * :576-646) or send it back to the star (re-emission of the same packet). */
enum { FS_NEW = 0, FS_EMIT, FS_RW, FS_TRACE, FS_ABSORB, FS_SCATTER, FS_DEAD, FS_NKIND };
/* outcome of a crossing */
enum { FX_CONT = 0, FX_INSIDE, FX_ESCAPE, FX_STAR, FX_GEOFAIL };

/* the current trace: optical depth to travel, travelled so far, crossings */
struct FTrace {
  double tau0, tau;
  int ntrace;
};

/* the per-cell accumulator updates of one crossing, applied by the caller
 * (directly, or aggregated over the lanes of a warp that share the cell) */
struct FDep {
  int c;       /* cell, -1 when nothing is deposited */
  int ni;      /* 1: the cell is not one of the packet's last two: exchange
                  lastphotnr and count the packet in Ni when another packet's
                  number was there (MCRadiation.f:943-946) */
  double ej;   /* EJv += */
  double ej2;  /* EJv2 += (cell exit only) */
};

TP_FN void f_apply_dep(const TAcc &A, size_t off, const FDep &d, int pid1) {
  if (d.c < 0) return;
  if (d.ni && tp_exch(&A.lastphot[off + d.c], pid1) != pid1) tp_addi(&A.Ni[off + d.c], 1);
  if (d.ej2 != 0.0) tp_add(&A.EJv2[off + d.c], d.ej2);
  tp_add(&A.EJv[off + d.c], d.ej);
}

/* accumulator offset of the sub-run packet pid belongs to (nruns) */
TP_FN size_t f_run_off(const TAcc &A, int64_t pid) { return (size_t)(pid / A.run_packets) * (size_t)A.ncell; }

template <class R>
TP_FN void f_packet_init(FPkt<R> &p, int64_t pid) {
  p.pid1 = (int)(pid + 1);
  p.q = p.u = p.v = (R)0;
  p.pol = 0;
  p.scatt = 0;
  p.cprev1 = p.cprev2 = -1;
}

/* star emission (MCRadiation.f:353-382) and the packet's first tau */
template <class R>
F_COLD void f_emit_star(const FModel<R> &m, px_stream *r, FPkt<R> &p, FTrace &t, TLocal &L) {
  p.nEJv = 0.0;
  (void)px_next(r); /* where_emit */
  R x, y, z;
  f_randomdirection<R>(r, &x, &y, &z);
  p.x = m.R0 * (double)x;
  p.y = m.R0 * (double)y;
  p.z = m.R0 * (double)z;
  L.cnt[TC_EMIT]++;
  {
    R ux, uy, uz;
    f_randomdirection<R>(r, &ux, &uy, &uz);
    f_set_dir<R>(p, ux, uy, uz);
  }
  p.scatt = 0;
  p.pol = 0;
  f_set_s<R>(p);
  {
    const double Lr = px_next(r) * m.Lstar;
    const int n = m.nlam - 1;
    int i = f_lower_bound(m.star_cdf, n, Lr);
    f_pick<R>(m, p, i, i < n ? m.star_cdf[i] : 0.0, i > 0 ? m.star_cdf[i - 1] : 0.0, Lr);
  }
  f_set_lambda<R>(m, p);
  p.E = m.Epkt;
  {
    R ux, uy, uz;
    f_randomdirection<R>(r, &ux, &uy, &uz);
    f_set_dir<R>(p, ux, uy, uz);
  }
  if (p.x * p.vx + p.y * p.vy + p.z * p.vz < 0.0) {
    p.vx = -p.vx;
    p.vy = -p.vy;
    p.vz = -p.vz;
  }
  p.edgeNr = 1;
  p.onEdge = 1;
  const double ct = fabs(p.z) / m.R0;
  p.i = 0;
  p.j = m.nt - 1;
  for (int j = 1; j <= m.nt - 1; ++j)
    if (ct >= m.Theta[j]) {
      p.j = j;
      break;
    }
  if (m.scattering) {
    p.pol = 0;
    p.scatt = 0;
    p.q = p.u = p.v = (R)0;
    f_set_s<R>(p);
  }
  t.tau0 = -log(px_next(r));
  t.tau = 0.0;
  t.ntrace = 0;
}

/* the state a trace starts in: the random walk first when the packet sits
 * inside a thick cell (MCRadiation.f:916) */
template <class R>
TP_FN int f_trace_state(const FModel<R> &m, const FPkt<R> &p) {
  return (m.rw && !p.onEdge && m.thick[p.i * m.nc + (p.j - 1)]) ? FS_RW : FS_TRACE;
}

/* SED bin of an escaping packet (MCRadiation.f:576-646) */
template <class R>
TP_FN void f_escape(const FModel<R> &m, const TAcc &A, const FPkt<R> &p, TLocal &L) {
  L.cnt[TC_ESCAPE]++;
  const double av = fabs(p.vz);
  int ia = (int)(av * (double)TP_NANG + 1.0);
  if (ia > TP_NANG) ia = TP_NANG;
  const int il = (p.wl1 > p.wl2) ? p.ilam1 : p.ilam1 + 1;
  const size_t k = (size_t)il * (TP_NANG + 1) + ia;
  const double wangle = 1.0 / ((double)ia / (double)TP_NANG - (double)(ia - 1) / (double)TP_NANG);
  const double add = ((wangle * p.E) * m.wlam[il]) / m.nruns_d;
  tp_add(&A.spec[k], add);
  tp_addi(&A.ispec[k], 1);
  if (p.scatt) tp_add(&A.scatspec[k], add);
}

/* one cell crossing of trace2d; the accumulator updates go to `d` */
template <class R>
TP_FN int f_cross(const FModel<R> &m, const TAcc &A, size_t off, FPkt<R> &p, FTrace &t, TLocal &L, FDep &d) {
  (void)A;
  (void)off;
  const int nlam = m.nlam;
  const int c = p.i * m.nc + (p.j - 1);
  /* Ni counts distinct packets per cell (lastphotnr, MCRadiation.f:943-946);
   * re-entering one of its last two cells, the packet's own number is
   * already there and the exchange is skipped */
  const bool recent = (c == p.cprev1) || (c == p.cprev2);
  if (!recent) {
    p.cprev2 = p.cprev1;
    p.cprev1 = c;
  }
  R kabs, kext;
  if (m.uniform_mix) {
    kabs = p.kabs;
    kext = m.scattering ? p.kext : p.kabs;
  } else {
    const R *Ka = m.KabsTotR + (size_t)c * nlam, *Ke = m.KextTotR + (size_t)c * nlam;
    kabs = Ka[p.ilam1] * p.wl1 + Ka[p.ilam1 + 1] * p.wl2;
    kext = m.scattering ? Ke[p.ilam1] * p.wl1 + Ke[p.ilam1 + 1] * p.wl2 : kabs;
  }
  double v;
  int inext, jnext;
  const int geo = f_trace2edge<R>(m, p, &v, &inext, &jnext);
  d.c = c;
  d.ni = !recent;
  d.ej = 0.0;
  d.ej2 = 0.0;
  if (geo) return FX_GEOFAIL;
  L.cnt[TC_CROSS]++;
  const double dAU = m.dens[c] * TP_AU;
  const double tau1 = ((double)kext * v) * dAU;
  if (t.tau + tau1 > t.tau0) {
    v = (v * (t.tau0 - t.tau)) / tau1;
    L.tautot += t.tau0 - t.tau;
    p.x += p.vx * v;
    p.y += p.vy * v;
    p.z += p.vz * v;
    p.onEdge = 0;
    const double dj = (p.E * v) * TP_AU * (double)kabs;
    d.ej = dj;
    p.nEJv += dj;
    /* the interaction's opacities at this point (Radiation.f:44-70) */
    p.kabs_i = kabs;
    p.ksca_i = kext - kabs;
    return FX_INSIDE;
  }
  p.x += p.vx * v;
  p.y += p.vy * v;
  p.z += p.vz * v;
  const double dj = (p.E * v) * TP_AU * (double)kabs;
  p.nEJv += dj;
  d.ej2 = p.nEJv * p.nEJv;
  p.nEJv = 0.0;
  d.ej = dj;
  p.onEdge = 1;
  t.tau += tau1;
  L.tautot += tau1;
  if (inext >= m.nr) return FX_ESCAPE;
  if (inext < 0) return FX_STAR;
  p.i = inext;
  p.j = jnext;
  if (++t.ntrace > m.nr * m.nt * 2) {
    L.cnt[TC_ABANDON]++;
    return FX_STAR;
  }
  return FX_CONT;
}

/* albedo test of an interaction (Radiation.f:74-76): FS_ABSORB or FS_SCATTER */
template <class R>
TP_FN int f_albedo(const FModel<R> &m, px_stream *r, FPkt<R> &p, TLocal &L) {
  typedef FOps<R> O;
  L.cnt[TC_INTERACT]++;
  if (!m.scattering) return FS_ABSORB;
  /* the non-uniform mixture's opacities at the interaction point are those
   * of the crossing that ended inside the cell; a uniform mixture's are the
   * packet's (kabs, kext - kabs).  Both give the reference's albedo. */
  R kabs, ksca;
  if (m.uniform_mix) {
    kabs = p.kabs;
    ksca = p.kext - p.kabs;
  } else {
    kabs = p.kabs_i;
    ksca = p.ksca_i;
  }
  const R albedo = ksca / (ksca + kabs);
  if (O::u(px_next(r)) > albedo) return FS_ABSORB;
  p.ksca_i = ksca;
  return FS_SCATTER;
}

/* absorption up to the wavelength draw: the cell's absorbed energy, the
 * temperatures before and after, the new direction and the draw xi.  What
 * the wavelength search needs is left in `a`. */
struct FAbs {
  int c, iT0, iT1;
  double e0, e1, T1, xi;
};

template <class R>
F_COLD void f_absorb_pre(const FModel<R> &m, const TAcc &A, size_t off, px_stream *r, FPkt<R> &p, TLocal &L,
                         FAbs &a) {
  const int c = p.i * m.nc + (p.j - 1);
  L.cnt[TC_ABSORB]++;
  if (A.Nabs) tp_addi(&A.Nabs[off + c], 1);
  p.scatt = 0;
  p.pol = 0;
  p.q = p.u = p.v = (R)0;
  const double *kp = m.KpCell + (m.uniform_mix ? (size_t)0 : (size_t)c * TP_TT);
  const double dE = p.E;
  const double Eold = tp_add(&A.Eabs[off + c], dE);
  const double mass = m.mass[c];
  int hint = A.kp_hint[off + c];
  int ib0, ib1;
  const double T0 = f_tinv(kp, Eold / mass, hint, &ib0, m.t4single);
  const double T1 = f_tinv(kp, (Eold + dE) / mass, ib0, &ib1, m.t4single);
  if (ib1 > hint) A.kp_hint[off + c] = ib1;
  int iT0 = (int)T0, iT1 = (int)T1;
  a.e0 = T0 - (double)iT0;
  a.e1 = T1 - (double)iT1;
  if (iT0 >= TP_TMAX - 1) iT0 = TP_TMAX - 2;
  if (iT1 >= TP_TMAX - 1) iT1 = TP_TMAX - 1;
  if (iT0 < 1) iT0 = 1;
  if (iT1 < 2) iT1 = 2;
  a.iT0 = iT0;
  a.iT1 = iT1;
  a.c = c;
  a.T1 = T1;
  /* new direction first (emit), then the wavelength draw */
  L.cnt[TC_EMIT]++;
  {
    R ux, uy, uz;
    f_randomdirection<R>(r, &ux, &uy, &uz);
    f_set_dir<R>(p, ux, uy, uz);
  }
  p.scatt = 0;
  p.pol = 0;
  f_set_s<R>(p);
  a.xi = px_next(r);
}

/* Re-emission spectrum of a uniform mixture as a cumulative over the nlam-1
 * trapezoid intervals: C(iT)[i] = cumulative of BB(iT) K, D(iT)[i] =
 * cumulative of (BB(iT+1) - BB(iT)) K, the (T0 -> T1) jump's cumulative is
 * [C(iT1) + e1 D(iT1)] - [C(iT0) + e0 D(iT0)], the reference's interpolated
 * Delta-B (Radiation.f:187-213) summed in the same order. */
template <class R>
struct FEmitU {
  const double *C0, *D0, *C1, *D1;
  double e0, e1;
  bool same;
  F_MFN double operator()(int i) const { return same ? D0[i] : (C1[i] + e1 * D1[i]) - (C0[i] + e0 * D0[i]); }
};

template <class R>
TP_FN FEmitU<R> f_emit_u(const FModel<R> &m, const FAbs &a) {
  const int n = m.nlam - 1;
  FEmitU<R> f;
  f.D0 = m.Dcum + (size_t)a.iT0 * n;
  f.C0 = m.Ccum + (size_t)a.iT0 * n;
  f.C1 = m.Ccum + (size_t)a.iT1 * n;
  f.D1 = m.Dcum + (size_t)a.iT1 * n;
  f.e0 = a.e0;
  f.e1 = a.e1;
  f.same = a.iT0 == a.iT1;
  return f;
}

/* A non-uniform mixture's re-emission spectrum at wavelength l: the
 * reference's spec(l) (Radiation.f:187-213) from the temperature-major
 * Planck rows and the cell's KabsTot row. */
template <class R>
struct FEmitN {
  const double *Ka, *P0, *P0p, *P1, *P1p;
  double e0, e1;
  bool same;
  F_MFN double operator()(int l) const {
    if (same) return (P0p[l] - P0[l]) * Ka[l];
    return (((e1 * P1p[l] + (1.0 - e1) * P1[l]) - e0 * P0p[l]) - (1.0 - e0) * P0[l]) * Ka[l];
  }
};

template <class R>
TP_FN FEmitN<R> f_emit_n(const FModel<R> &m, const FAbs &a, double *Lr) {
  const int nlam = m.nlam;
  FEmitN<R> f;
  f.Ka = m.KabsTot + (size_t)a.c * nlam;
  f.P0 = m.BBT + (size_t)a.iT0 * nlam;
  f.P0p = f.P0 + nlam;
  f.P1 = m.BBT + (size_t)a.iT1 * nlam;
  f.P1p = f.P1 + nlam;
  f.e0 = a.e0;
  f.e1 = a.e1;
  f.same = a.iT0 == a.iT1;
  const double *kp = m.KpCell + (size_t)a.c * TP_TT;
  const int i0 = a.iT0, i1 = a.iT1;
  const double e0 = a.e0, e1 = a.e1;
  const double kpe = i0 == i1 ? kp[i0 + 1] - kp[i0]
                              : ((e1 * kp[i1 + 1] + (1.0 - e1) * kp[i1]) - e0 * kp[i0 + 1]) - (1.0 - e0) * kp[i0];
  *Lr = a.xi * kpe;
  return f;
}

/* the wavelength search of one lane on its own */
template <class R>
F_COLD void f_absorb_search(const FModel<R> &m, FPkt<R> &p, const FAbs &a) {
  const int n = m.nlam - 1;
  if (m.uniform_mix) {
    const FEmitU<R> f = f_emit_u<R>(m, a);
    const double tot = f(n - 1);
    const double Lr = a.xi * tot;
    int i;
    if (f.same) {
      int gk = (int)(a.xi * (double)F_NGUIDE);
      if (gk > F_NGUIDE - 1) gk = F_NGUIDE - 1;
      i = f_walk([&](int k) { return f.D0[k]; }, n, (int)m.emitG[(size_t)a.iT0 * F_NGUIDE + gk], Lr, true);
    } else {
      int lo = 0, hi = n;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (f(mid) >= Lr)
          hi = mid;
        else
          lo = mid + 1;
      }
      i = lo;
    }
    f_pick<R>(m, p, i, i < n ? f(i) : 0.0, i > 0 ? f(i - 1) : 0.0, Lr);
  } else {
    /* sequential scan (Radiation.f:187-213), the additions in the
     * reference's order; eight wavelengths' loads are issued together */
    double Lr;
    const FEmitN<R> spec = f_emit_n<R>(m, a, &Lr);
    double Lt = 0.0, Ltold = 0.0, s0 = spec(0);
    int i = n;
    for (int i0 = 0; i0 < n && i == n; i0 += 8) {
      double sb[8], dn[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int l = i0 + u;
        sb[u] = l < n ? spec(l + 1) : 0.0;
        dn[u] = l < n ? m.dnu_half[l] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (i0 + u >= n) break;
        Lt = Lt + dn[u] * (s0 + sb[u]);
        if (Lt >= Lr) {
          i = i0 + u;
          break;
        }
        Ltold = Lt;
        s0 = sb[u];
      }
    }
    f_pick<R>(m, p, i, Lt, Ltold, Lr);
  }
}

template <class R>
TP_FN void f_absorb_post(const FModel<R> &m, const TAcc &A, size_t off, FPkt<R> &p, const FAbs &a) {
  f_set_lambda<R>(m, p);
  A.T[off + a.c] = a.T1;
}

/* scattering up to the component pick (Radiation.f:259-290): isotropic
 * scattering is complete here (returns -1 with the new direction set);
 * otherwise returns 1 and leaves the draw KscaR for the pick */
template <class R>
TP_FN int f_scatter_pre(const FModel<R> &m, px_stream *r, FPkt<R> &p, TLocal &L, R *KscaR) {
  typedef FOps<R> O;
  L.cnt[TC_SCATTER]++;
  p.scatt = 1;
  if (m.scat_how == 1) {
    R ux, uy, uz;
    f_randomdirection<R>(r, &ux, &uy, &uz);
    f_set_dir<R>(p, ux, uy, uz);
    return -1;
  }
  *KscaR = O::u(px_next(r)) * p.ksca_i;
  return 1;
}

/* the component and wavelength end whose scattering matrix is used: the
 * reference's order (Radiation.f:273-290), per component the l1+1 term,
 * then the l1 term; -1 - (fallback material) when the draw exceeds the sum
 * (the averaged-matrix branch, :293-315) */
template <class R>
TP_FN int f_scatter_pick(const FModel<R> &m, const FPkt<R> &p, R KscaR) {
  const int nlam = m.nlam, l1 = p.ilam1;
  const int c = p.i * m.nc + (p.j - 1);
  const double *w = m.comp_w + (size_t)c * m.ncomp;
  int mat = -1, qlast = 0, llast = l1;
  for (int q0 = 0; q0 < m.ncomp && mat < 0; q0 += 4) {
    R w2b[4], w1b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = q0 + u;
      const R wq = q < m.ncomp ? (R)w[q] : (R)0;
      w2b[u] = q < m.ncomp ? wq * p.wl2 * m.Ksca_c[q * nlam + l1 + 1] : (R)0;
      w1b[u] = q < m.ncomp ? wq * p.wl1 * m.Ksca_c[q * nlam + l1] : (R)0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = q0 + u;
      if (q >= m.ncomp) break;
      KscaR -= w2b[u];
      if (KscaR < (R)0) {
        mat = q * nlam + l1 + 1;
        break;
      }
      KscaR -= w1b[u];
      if (KscaR < (R)0) {
        mat = q * nlam + l1;
        break;
      }
      if (w2b[u] > (R)0) { qlast = q; llast = l1 + 1; }
      if (w1b[u] > (R)0) { qlast = q; llast = l1; }
    }
  }
  if (mat < 0) return -1 - (qlast * nlam + llast);
  return mat;
}

/* the scattering matrix's use of the pick: the averaged-matrix counter and
 * the new direction and Stokes vector (Radiation.f:381-495) */
template <class R>
TP_FN void f_scatter_post(const FModel<R> &m, px_stream *r, FPkt<R> &p, TLocal &L, int pick) {
  if (pick < 0) {
    L.cnt[TC_AVGMAT]++;
    pick = -1 - pick;
  }
  f_scatangle<R>(m, r, p, pick);
}

/* the overflow roulette (MCRadiation.f:568-571) and the next tau (:573);
 * returns 0 when the roulette ends the packet */
template <class R>
TP_FN int f_after_interact(const FModel<R> &m, px_stream *r, FPkt<R> &p, FTrace &t, TLocal &L) {
  if (m.maxinteract > 0) {
    if (px_next(r) < 1.0 / (double)m.maxinteract) {
      L.cnt[TC_OVERFLOW]++;
      return 0;
    }
    p.E = (p.E * (double)m.maxinteract) / (double)(m.maxinteract - 1);
  }
  t.tau0 = -log(px_next(r));
  t.tau = 0.0;
  t.ntrace = 0;
  return 1;
}

/* ------------------------------------------------------------- random walk */
/* one jump of the modified random walk (RandomWalk.f:15-147); returns 1
 * when the packet jumped (then a new outward direction follows) */
template <class R>
F_COLD int f_random_walk(const FModel<R> &m, const TAcc &A, size_t off, px_stream *r, FPkt<R> &p, TLocal &L) {
  const int c = p.i * m.nc + (p.j - 1);
  /* distance to the nearest face (MinDist, RandomWalk.f:15-43) */
  double rho = p.x * p.x + p.y * p.y;
  const double rr = sqrt(rho + p.z * p.z);
  rho = sqrt(rho);
  const double z = fabs(p.z);
  double dmin = fabs(rr - m.Rr[p.i]);
  double t = fabs(m.Rr[p.i + 1] - rr);
  if (t < dmin) dmin = t;
  t = fabs(m.Theta[p.j - 1] * rho - m.SinTheta[p.j - 1] * z);
  if (t < dmin) dmin = t;
  t = fabs(m.Theta[p.j] * rho - m.SinTheta[p.j] * z);
  if (t < dmin) dmin = t;
  /* no jump at any temperature: dmin is within factRW of the cell's
   * shortest mean free path (the test below at the current temperature
   * would fail too), so the table lookups are skipped */
  if (m.rw_dmin && dmin <= m.rw_dmin[c]) return 0;
  const int row = m.kd_index[c];
  if (row < 0) return 0;
  int iT = (int)A.T[off + c];
  if (iT < 1) iT = 1;
  if (iT > TP_TMAX - 1) iT = TP_TMAX - 1;
  const double Kext = m.KDext[(size_t)row * TP_TT + iT];
  const double lr = 1.0 / ((TP_AU * Kext) * m.dens[c]);
  if (dmin <= m.factRW * lr) return 0;
  int iy = 1;
  tp_hunt(m.rw_phi, TP_NY, px_next(r), &iy);
  const double v = ((-3.0 * m.rw_logy[iy - 1]) * (dmin * dmin)) / (lr * (TP_PI * TP_PI));
  const double Kabs = m.KDabs[(size_t)row * TP_TT + iT];
  R ux, uy, uz;
  f_randomdirection<R>(r, &ux, &uy, &uz);
  f_set_dir<R>(p, ux, uy, uz);
  p.x += dmin * p.vx;
  p.y += dmin * p.vy;
  p.z += dmin * p.vz;
  const double EJv = (p.E * v) * TP_AU;
  const double dEa = (EJv * Kabs) * m.dens[c];
  const double Eold = tp_add(&A.Eabs[off + c], dEa);
  tp_add(&A.EJv[off + c], EJv * Kabs);
  p.nEJv += EJv * Kabs;
  const double *kp = m.KpCell + (m.uniform_mix ? (size_t)0 : (size_t)c * TP_TT);
  int ib;
  A.T[off + c] = f_tinv(kp, (Eold + dEa) / m.mass[c], A.kp_hint[off + c], &ib, m.t4single);
  if (ib > A.kp_hint[off + c]) A.kp_hint[off + c] = ib;
  L.tautot += v / dmin;
  L.cnt[TC_RWSTEP]++;
  return 1;
}

/* the new direction after a jump: outward from the jump (RandomWalk.f) */
template <class R>
TP_FN void f_rw_redirect(px_stream *r, FPkt<R> &p) {
  R vx, vy, vz;
  do {
    f_randomdirection<R>(r, &vx, &vy, &vz);
  } while ((R)p.vx * vx + (R)p.vy * vy + (R)p.vz * vz < (R)0);
  f_set_dir<R>(p, vx, vy, vz);
}

/* ------------------------------------------------------------- one packet */
/* One packet as a state machine: f_slot_start sets it up, f_slot_step
 * advances it by one event (accumulators updated directly) and returns 1
 * when the packet has ended. */
template <class R>
struct FSlot {
  FPkt<R> p;
  px_stream rs;
  FTrace t;
  size_t off;
  int st;
};

template <class R>
TP_FN void f_slot_start(const FModel<R> &m, const TAcc &A, FSlot<R> &s, int64_t pid) {
  s.off = f_run_off(A, pid);
  px_init(&s.rs, m.seed, (uint64_t)pid);
  f_packet_init<R>(s.p, pid);
  s.st = FS_EMIT;
}

template <class R>
TP_FN int f_slot_step(const FModel<R> &m, const TAcc &A, FSlot<R> &s, TLocal &L) {
  FPkt<R> &p = s.p;
  px_stream *r = &s.rs;
  if (s.st == FS_EMIT) {
    f_emit_star<R>(m, r, p, s.t, L);
    s.st = FS_TRACE; /* on the star's surface: never inside a thick cell */
  } else if (s.st == FS_RW) {
    if (f_random_walk<R>(m, A, s.off, r, p, L))
      f_rw_redirect<R>(r, p);
    else
      s.st = FS_TRACE;
  } else if (s.st == FS_TRACE) {
    FDep d;
    const int o = f_cross<R>(m, A, s.off, p, s.t, L, d);
    f_apply_dep(A, s.off, d, p.pid1);
    if (o == FX_INSIDE) {
      s.st = f_albedo<R>(m, r, p, L);
    } else if (o == FX_ESCAPE) {
      f_escape<R>(m, A, p, L);
      return 1;
    } else if (o == FX_STAR) {
      L.cnt[TC_HITSTAR]++;
      s.st = FS_EMIT;
    } else if (o == FX_GEOFAIL) {
      L.cnt[TC_GEOFAIL]++;
      return 1;
    }
  } else {
    if (s.st == FS_ABSORB) {
      FAbs a;
      f_absorb_pre<R>(m, A, s.off, r, p, L, a);
      f_absorb_search<R>(m, p, a);
      f_absorb_post<R>(m, A, s.off, p, a);
    } else {
      R KscaR;
      if (f_scatter_pre<R>(m, r, p, L, &KscaR) > 0) f_scatter_post<R>(m, r, p, L, f_scatter_pick<R>(m, p, KscaR));
    }
    if (!f_after_interact<R>(m, r, p, s.t, L)) return 1;
    s.st = f_trace_state<R>(m, p);
  }
  return 0;
}

/* All events of one packet back to back: the host replay of the device code
 * and the batched kernel. */
template <class R>
TP_FN void f_run_packet(const FModel<R> &m, const TAcc &A, int64_t pid, TLocal &L) {
  FSlot<R> s;
  f_slot_start<R>(m, A, s, pid);
  while (!f_slot_step<R>(m, A, s, L)) {
  }
}

#endif /* MCMAX_TRANSPORT_FAST_CUH */
