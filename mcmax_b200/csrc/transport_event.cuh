/*
 * transport_event.cuh -- the single-model packet loop as a warp scheduler
 * over packet events (device code).
 *
 * Each lane of a persistent warp owns one packet (its state in registers)
 * and the packet moves through the events of transport_fast.cuh: emission,
 * random-walk jump, cell crossing, absorption, scattering.  The warp does
 * not let every lane run its own control flow (lanes in a crossing loop
 * would idle while one lane absorbs, and the reverse); it counts the lanes
 * waiting for each event kind (ballots) and executes one kind at a time for
 * all lanes that wait for it, the kind with the most lanes first.  A
 * crossing phase runs crossing after crossing while the crossing lanes are
 * still the largest group.  When a packet ends, its lane takes the next
 * packet id from the work counter (one atomic per warp).
 *
 * Searches over tables (the re-emission wavelength, the scattering
 * component of a settled mixture) run warp-cooperatively when few lanes
 * need them: all 32 lanes probe 32 table positions of one lane's search at
 * once, which turns a binary search of 8 dependent loads into 2 rounds and
 * a wavelength scan over nlam entries into nlam/32 rounds of a warp prefix
 * sum.  That is what shortens the tail of a run, where a few trapped
 * packets are alone in their warps.
 *
 * Per-cell deposits of a crossing step (EJv, EJv2) can be combined over the
 * lanes that sit in the same cell (__match_any_sync on the cell) and written
 * with one atomic per cell (FE_AGGREGATE=1).  Measured on the precision deck
 * it does not pay: atomics on the cell accumulators are not contended enough,
 * and the match and the group sums cost more than they save (the bulk of a
 * 1e7-packet run is about 10 % faster with plain per-lane atomics), so it is
 * off by default.  The lastphotnr exchange of a crossing
 * (MCRadiation.f:943-946) is issued at once and its answer read at the
 * packet's next crossing, so its round trip overlaps the next crossing's
 * arithmetic.
 */
#ifndef MCMAX_TRANSPORT_EVENT_CUH
#define MCMAX_TRANSPORT_EVENT_CUH

#include "transport_fast.cuh"

#define FE_FULL 0xffffffffu

/* at most this many lanes in a search phase: cooperative searches, one lane
 * after the other; more: every lane searches on its own */
#ifndef FE_COOP_MAX
#define FE_COOP_MAX 4
#endif
/* a crossing phase continues while FE_TRACE_KEEP x (crossing lanes) is at
 * least the largest group of lanes waiting for another event: crossings are
 * cheap and interactions dear, so letting more lanes gather for an
 * interaction pays (1e8 packets, settled deck: the bulk of the run 7 %
 * shorter with 2 than with 1; 4 is slower again) */
#ifndef FE_TRACE_KEEP
#define FE_TRACE_KEEP 2
#endif
/* 1: combine same-cell deposits of a crossing step within the warp */
#ifndef FE_AGGREGATE
#define FE_AGGREGATE 0
#endif

/* first i in [0,n) with f(i) >= v (ge) or f(i) > v, n when none; f is
 * non-decreasing and is evaluated by all 32 lanes at once (ceil(log32 n)
 * rounds).  Warp-uniform arguments, called by the full warp. */
template <class F>
__device__ __forceinline__ int fe_lower_bound(const F &f, int n, double v, bool ge, int lane) {
  int lo = 0, len = n;
  while (len > 32) {
    const int S = (len + 31) >> 5;
    int pidx = lo + (lane + 1) * S - 1;
    if (pidx > lo + len - 1) pidx = lo + len - 1;
    const double fv = f(pidx);
    const unsigned hit = __ballot_sync(FE_FULL, ge ? fv >= v : fv > v);
    if (!hit) return n; /* only at the top level: deeper, the segment's last probe hit */
    const int j = __ffs(hit) - 1;
    const int seg_lo = lo + j * S;
    int seg_hi = lo + (j + 1) * S - 1;
    if (seg_hi > lo + len - 1) seg_hi = lo + len - 1;
    lo = seg_lo;
    len = seg_hi - seg_lo + 1;
  }
  bool h = false;
  if (lane < len) {
    const double fv = f(lo + lane);
    h = ge ? fv >= v : fv > v;
  }
  const unsigned hit = __ballot_sync(FE_FULL, h);
  return hit ? lo + __ffs(hit) - 1 : n;
}

/* The trapezoid cumulative Lt(i) = sum_{k<=i} dn[k] (s(k) + s(k+1)) over the
 * intervals i in [0,n) of a spectrum s (n+1 points), 32 intervals per round
 * with a warp prefix sum; returns the first i with Lt(i) >= Lr (n when
 * none) with Lt(i) and Lt(i-1) (0 before the first interval). */
template <class S>
__device__ __forceinline__ int fe_scan(const S &s, const double *dn, int n, double Lr, int lane, double *Lt_out,
                                       double *Ltold_out) {
  double carry = 0.0;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const int li = i < n ? i : n;
    const double si = s(li);
    double sn = __shfl_down_sync(FE_FULL, si, 1);
    if (lane == 31) sn = s(base + 32 < n ? base + 32 : n);
    double x = i < n ? dn[i] * (si + sn) : 0.0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const double y = __shfl_up_sync(FE_FULL, x, d);
      if (lane >= d) x += y;
    }
    const double Lt = carry + x;
    const unsigned hit = __ballot_sync(FE_FULL, i < n && Lt >= Lr);
    if (hit) {
      const int j = __ffs(hit) - 1;
      const double a = __shfl_sync(FE_FULL, Lt, j);
      const double b = __shfl_sync(FE_FULL, Lt, j > 0 ? j - 1 : 0);
      *Lt_out = a;
      *Ltold_out = j > 0 ? b : carry;
      return base + j;
    }
    carry = __shfl_sync(FE_FULL, Lt, 31);
  }
  *Lt_out = carry;
  *Ltold_out = carry;
  return n;
}

/* The scattering component pick of one packet (Radiation.f:273-290), 32
 * components per round: component q contributes w_q wl2 Ksca_q(l1+1), then
 * w_q wl1 Ksca_q(l1); the first term whose running sum exceeds the draw
 * KscaR picks (component, wavelength end).  Same result as f_scatter_pick
 * up to the order of the additions. */
template <class R>
__device__ __forceinline__ int fe_scatter_pick(const FModel<R> &m, int c, int l1, R wl1, R wl2, R KscaR, int lane) {
  const int nlam = m.nlam, ncomp = m.ncomp;
  const double *w = m.comp_w + (size_t)c * ncomp;
  R carry = (R)0;
  int qlast = 0, llast = l1;
  for (int base = 0; base < ncomp; base += 32) {
    const int q = base + lane;
    R w2b = (R)0, w1b = (R)0;
    if (q < ncomp) {
      const R wq = (R)w[q];
      w2b = wq * wl2 * m.Ksca_c[q * nlam + l1 + 1];
      w1b = wq * wl1 * m.Ksca_c[q * nlam + l1];
    }
    R x = w2b + w1b;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const R y = __shfl_up_sync(FE_FULL, x, d);
      if (lane >= d) x += y;
    }
    const R before = carry + (x - (w2b + w1b));
    const bool h2 = q < ncomp && before + w2b > KscaR;
    const bool h1 = q < ncomp && before + w2b + w1b > KscaR;
    const unsigned hit = __ballot_sync(FE_FULL, h2 || h1);
    if (hit) {
      const int j = __ffs(hit) - 1;
      const bool second = __shfl_sync(FE_FULL, h2 ? 1 : 0, j) != 0;
      return (base + j) * nlam + (second ? l1 + 1 : l1);
    }
    const unsigned pos = __ballot_sync(FE_FULL, q < ncomp && (w2b > (R)0 || w1b > (R)0));
    if (pos) {
      const int jl = 31 - __clz(pos);
      const bool one = __shfl_sync(FE_FULL, w1b > (R)0 ? 1 : 0, jl) != 0;
      qlast = base + jl;
      llast = one ? l1 : l1 + 1;
    }
    carry = __shfl_sync(FE_FULL, carry + x, 31);
  }
  return -1 - (qlast * nlam + llast);
}

/* EJv / EJv2 of one crossing step, combined over the lanes in the same cell:
 * one atomic per distinct cell.  Called by the full warp. */
__device__ __forceinline__ void fe_deposit(const TAcc &A, size_t off, const FDep &d, int lane) {
#if FE_AGGREGATE
  const bool has = d.c >= 0;
  const unsigned long long key = has ? (unsigned long long)(off + (size_t)d.c) : ~0ULL - (unsigned long long)lane;
  const unsigned g = __match_any_sync(FE_FULL, key);
  if (!has) return;
  double ej = d.ej, ej2 = d.ej2;
  if (g != (1u << lane)) {
    double s1 = 0.0, s2 = 0.0;
    for (unsigned mm = g; mm; mm &= mm - 1) {
      const int src = __ffs(mm) - 1;
      s1 += __shfl_sync(g, ej, src);
      s2 += __shfl_sync(g, ej2, src);
    }
    ej = s1;
    ej2 = s2;
  }
  if (lane == __ffs(g) - 1) {
    atomicAdd(&A.EJv[key], ej);
    if (ej2 != 0.0) atomicAdd(&A.EJv2[key], ej2);
  }
#else
  (void)lane;
  if (d.c < 0) return;
  if (d.ej2 != 0.0) atomicAdd(&A.EJv2[off + d.c], d.ej2);
  atomicAdd(&A.EJv[off + d.c], d.ej);
#endif
}

/* phase statistics kept in the free counter slots 12..15, counted while all
 * 32 lanes of the warp hold packets */
enum { TC_PHASES = 12, TC_PHASE_LANES = 13, TC_XSTEPS = 14, TC_XLANES = 15 };

template <class R>
__device__ void fe_event_loop(const FModel<R> &m, const TAcc &A, TLocal &L) {
  const int lane = threadIdx.x & 31;
  FPkt<R> p;
  p.pid1 = 0;
  px_stream rs;
  FTrace t;
  FAbs a;
  size_t off = 0;
  int st = FS_NEW;
  int pend_c = -1, pend_prev = 0; /* lastphotnr exchange in flight */
  const int n1 = m.nlam - 1;
  const unsigned long long t0 = tp_globaltimer();
  unsigned iter = 0;
  /* the pending Ni update of the last crossing */
  auto resolve_ni = [&]() {
    if (pend_c >= 0) {
      if (pend_prev != p.pid1) atomicAdd(&A.Ni[off + pend_c], 1);
      pend_c = -1;
    }
  };
  auto finish = [&]() {
    resolve_ni();
    tp_packet_done(A);
    st = FS_NEW;
  };
  for (;;) {
    /* lanes without a packet take the next ids */
    const unsigned mnew = __ballot_sync(FE_FULL, st == FS_NEW);
    if (mnew) {
      const int leader = __ffs(mnew) - 1;
      unsigned long long base = 0ULL;
      if (lane == leader) base = atomicAdd(A.next, (unsigned long long)__popc(mnew));
      base = __shfl_sync(FE_FULL, base, leader);
      if (m.maxruntime > 0.0) {
        /* a run stopped by maxruntime is discarded whole: the warp leaves */
        int stop = 0;
        if (lane == leader)
          stop = base < (unsigned long long)m.nphot && tp_runtime_stop(A, m.maxruntime, m.nphot, base, t0);
        if (__shfl_sync(FE_FULL, stop, leader)) break;
      }
      if (st == FS_NEW) {
        const unsigned long long k = base + (unsigned long long)__popc(mnew & ((1u << lane) - 1u));
        if (k >= (unsigned long long)m.nphot) {
          st = FS_DEAD;
        } else {
          const int64_t pid = (int64_t)k + m.pid0;
          off = f_run_off(A, pid);
          px_init(&rs, m.seed, (uint64_t)pid);
          f_packet_init<R>(p, pid);
          st = FS_EMIT;
        }
      }
    }
    if (m.maxruntime > 0.0 && (++iter & 63u) == 0u) {
      int stop = 0;
      if (lane == 0) stop = *(volatile unsigned long long *)A.stop != 0ULL;
      if (__shfl_sync(FE_FULL, stop, 0)) break;
    }
    const unsigned mE = __ballot_sync(FE_FULL, st == FS_EMIT);
    const unsigned mR = __ballot_sync(FE_FULL, st == FS_RW);
    const unsigned mT = __ballot_sync(FE_FULL, st == FS_TRACE);
    const unsigned mA = __ballot_sync(FE_FULL, st == FS_ABSORB);
    const unsigned mS = __ballot_sync(FE_FULL, st == FS_SCATTER);
    if (!(mE | mR | mT | mA | mS)) break;
    int kind = FS_TRACE, best = __popc(mT);
    if (__popc(mA) > best) { kind = FS_ABSORB; best = __popc(mA); }
    if (__popc(mS) > best) { kind = FS_SCATTER; best = __popc(mS); }
    if (__popc(mR) > best) { kind = FS_RW; best = __popc(mR); }
    if (__popc(mE) > best) { kind = FS_EMIT; best = __popc(mE); }
    /* phase statistics of full warps only (every lane holds a packet): the
     * lane efficiency of the bulk of the run, not of its tail */
    const bool full = (mE | mR | mT | mA | mS) == FE_FULL;
    if (lane == 0 && full) {
      L.cnt[TC_PHASES]++;
      L.cnt[TC_PHASE_LANES] += (unsigned)best;
    }
    if (kind == FS_TRACE) {
      unsigned mt = mT;
      for (;;) {
        FDep d;
        d.c = -1;
        int o = FX_CONT;
        if (st == FS_TRACE) {
          resolve_ni();
          o = f_cross<R>(m, A, off, p, t, L, d);
          if (d.ni) {
            pend_prev = atomicExch(&A.lastphot[off + d.c], p.pid1);
            pend_c = d.c;
          }
        }
        fe_deposit(A, off, d, lane);
        if (lane == 0 && full) {
          L.cnt[TC_XSTEPS]++;
          L.cnt[TC_XLANES] += (unsigned)__popc(mt);
        }
        if (st == FS_TRACE && o != FX_CONT) {
          if (o == FX_INSIDE) {
            st = f_albedo<R>(m, &rs, p, L);
          } else if (o == FX_ESCAPE) {
            f_escape<R>(m, A, p, L);
            finish();
          } else if (o == FX_STAR) {
            L.cnt[TC_HITSTAR]++;
            st = FS_EMIT;
          } else {
            L.cnt[TC_GEOFAIL]++;
            finish();
          }
        }
        mt = __ballot_sync(FE_FULL, st == FS_TRACE);
        if (!mt) break;
        /* keep crossing while the crossing lanes are the largest group */
        const int nt = __popc(mt);
        if (nt < 32) {
          const int others = max(max(__popc(__ballot_sync(FE_FULL, st == FS_ABSORB)),
                                     __popc(__ballot_sync(FE_FULL, st == FS_SCATTER))),
                                 __popc(__ballot_sync(FE_FULL, st == FS_EMIT || st == FS_NEW || st == FS_RW)));
          if (nt * FE_TRACE_KEEP < others) break;
        }
      }
    } else if (kind == FS_ABSORB) {
      const bool me = st == FS_ABSORB;
      if (me) f_absorb_pre<R>(m, A, off, &rs, p, L, a);
      if (m.uniform_mix && __popc(mA) > FE_COOP_MAX) {
        if (me) f_absorb_search<R>(m, p, a);
      } else {
        /* one lane's search at a time, all lanes probing */
        for (unsigned mm = mA; mm; mm &= mm - 1) {
          const int o = __ffs(mm) - 1;
          FAbs b;
          b.c = __shfl_sync(FE_FULL, a.c, o);
          b.iT0 = __shfl_sync(FE_FULL, a.iT0, o);
          b.iT1 = __shfl_sync(FE_FULL, a.iT1, o);
          b.e0 = __shfl_sync(FE_FULL, a.e0, o);
          b.e1 = __shfl_sync(FE_FULL, a.e1, o);
          b.xi = __shfl_sync(FE_FULL, a.xi, o);
          int i;
          double Lt, Ltold, Lr;
          if (m.uniform_mix) {
            const FEmitU<R> f = f_emit_u<R>(m, b);
            Lr = b.xi * f(n1 - 1);
            i = fe_lower_bound(f, n1, Lr, true, lane);
            Lt = 0.0;
            Ltold = 0.0;
            if (lane == o) {
              Lt = i < n1 ? f(i) : 0.0;
              Ltold = i > 0 ? f(i - 1) : 0.0;
            }
          } else {
            const FEmitN<R> s = f_emit_n<R>(m, b, &Lr);
            i = fe_scan(s, m.dnu_half, n1, Lr, lane, &Lt, &Ltold);
          }
          if (lane == o) f_pick<R>(m, p, i, Lt, Ltold, Lr);
        }
      }
      if (me) {
        f_absorb_post<R>(m, A, off, p, a);
        if (f_after_interact<R>(m, &rs, p, t, L))
          st = f_trace_state<R>(m, p);
        else
          finish();
      }
    } else if (kind == FS_SCATTER) {
      const bool me = st == FS_SCATTER;
      R KscaR = (R)0;
      int go = 0;
      if (me) go = f_scatter_pre<R>(m, &rs, p, L, &KscaR);
      const unsigned mp = __ballot_sync(FE_FULL, go > 0);
      int pick = 0;
      if (mp) {
        if (m.uniform_mix && __popc(mp) > FE_COOP_MAX) {
          if (go > 0) pick = f_scatter_pick<R>(m, p, KscaR);
        } else {
          for (unsigned mm = mp; mm; mm &= mm - 1) {
            const int o = __ffs(mm) - 1;
            const int c = __shfl_sync(FE_FULL, p.i * m.nc + (p.j - 1), o);
            const int l1 = __shfl_sync(FE_FULL, p.ilam1, o);
            const R wl1 = __shfl_sync(FE_FULL, p.wl1, o);
            const R wl2 = __shfl_sync(FE_FULL, p.wl2, o);
            const R kr = __shfl_sync(FE_FULL, KscaR, o);
            const int pk = fe_scatter_pick<R>(m, c, l1, wl1, wl2, kr, lane);
            if (lane == o) pick = pk;
          }
        }
      }
      if (go > 0) f_scatter_post<R>(m, &rs, p, L, pick);
      if (me) {
        if (f_after_interact<R>(m, &rs, p, t, L))
          st = f_trace_state<R>(m, p);
        else
          finish();
      }
    } else if (kind == FS_RW) {
      if (st == FS_RW) {
        if (f_random_walk<R>(m, A, off, &rs, p, L))
          f_rw_redirect<R>(&rs, p);
        else
          st = FS_TRACE;
      }
    } else {
      if (st == FS_EMIT) {
        f_emit_star<R>(m, &rs, p, t, L);
        st = FS_TRACE;
      }
    }
  }
}

#endif /* MCMAX_TRANSPORT_EVENT_CUH */
