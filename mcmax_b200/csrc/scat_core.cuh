/*
 * scat_core.cuh -- the scattered-light field of the ray tracer: the second
 * Monte Carlo of TraceMono (TraceMono.f:583-914) and the pieces it calls,
 * shared by the library's kernels (scatfield.cu, raytrace.cu).
 *
 *   sub-cells      each theta row j of a full-Mueller field is split into
 *                  nrg = int((thet(j+1) - thet(j)) 270 / pi) cones (at least
 *                  1), with cos^2 edges thetrg (Telescope.f:93-110); the
 *                  field and the ray paths carry the sub-cell index irg
 *   sf_trace2edge_rg  Trace2edgeRG (TraceMono.f:2487-2657): the cell-edge
 *                  step of the packet loop with the sub-cones as extra
 *                  theta edges
 *   sf_cell_*      the cell's extinction, albedo and mixed Mueller matrix at
 *                  the wavelength (TraceMono.f:664-750), the thermal
 *                  emission weight of EmissionDistribution (TraceMono.f:
 *                  1005-1057, thermal contact) and the shortest absorption
 *                  depth to the outside over nexits directions
 *                  (TraceMono.f:1076-1105, trace2exit TraceMono.f:2659-2697)
 *   field layout   SF[((i nsub + off[j-1] + irg - 1) 2 + side) 91 + b]: ring
 *                  i, sub-cell irg of row j, side 0 above the midplane (the
 *                  reference's side 1), bin b = 0 the total E v AU and bins
 *                  1..90 the intensity towards the observer directions that
 *                  makescattfield folds onto half a circle
 *                  (TraceMono.f:1430-1497); for isotropic scattering one
 *                  sub-cell per cell and only bin 0 is used
 *   sf_jphi        the folded azimuth bin of a path point (trace2dpath,
 *                  TraceMono.f:2378-2400)
 *
 * The packets themselves (MakeStarScatter, emitposition, trace2dmono,
 * makescattfield and the albedo roulette) are written as warp-cooperative
 * kernels in scatfield.cu.
 */
#ifndef MCMAX_SCAT_CORE_CUH
#define MCMAX_SCAT_CORE_CUH

#include <math.h>
#include <stddef.h>

#include <vector>

#include "transport_core.cuh"

#ifdef __CUDACC__
#define SF_HD __host__ __device__ inline
#else
#define SF_HD static inline
#endif

#define SF_NPHI 180             /* NPHISCATT (Modules.f:6) */
#define SF_NB (SF_NPHI / 2 + 1) /* bins 0..90 of one side of a sub-cell */

/* the sub-cell grid in theta */
struct SfGeom {
  int nsub;               /* sub-cells of one ring: the sum of nrg over the rows */
  const int *nrg;         /* nt-1: sub-cells of row j at [j-1] */
  const int *off;         /* nt-1: first sub-cell of row j within a ring */
  const double *thetrg;   /* nsub + nt-1: row j's nrg+1 cos^2 edges from off[j-1] + j-1 */
  const double *fracirg;  /* nsub: the sub-cell's share of the row's cos theta range */
};

/* host: the sub-cell tables of Telescope.f:93-110 and TraceMono.f:321-328.
 * thet: the nt polar edges; Theta: their cosines.  The first and last edge
 * of a row are the row's own Theta^2, which is what cos(thet)^2 gives
 * there. */
struct SfGeomHost {
  std::vector<int> nrg, off;
  std::vector<double> thetrg, fracirg;
  int nsub = 0;
};

static inline void sf_geom_build(int nt, const double *thet, const double *Theta, bool angular, SfGeomHost *g) {
  const int nc = nt - 1;
  g->nrg.assign(nc, 1);
  g->off.assign(nc, 0);
  int n = 0;
  for (int j = 1; j <= nc; ++j) {
    int k = 1;
    if (angular) {
      const int q = (int)((thet[j] - thet[j - 1]) * 270.0 / TP_PI);
      if (q > 1) k = q;
    }
    g->nrg[j - 1] = k;
    g->off[j - 1] = n;
    n += k;
  }
  g->nsub = n;
  g->thetrg.assign((size_t)n + nc, 0.0);
  g->fracirg.assign((size_t)n, 0.0);
  for (int j = 1; j <= nc; ++j) {
    const int k = g->nrg[j - 1];
    double *tr = &g->thetrg[(size_t)g->off[j - 1] + (j - 1)];
    const double dth = (thet[j] - thet[j - 1]) / (double)(float)k;
    for (int q = 1; q <= k + 1; ++q) {
      const double c = cos(thet[j - 1] + (double)(float)(q - 1) * dth);
      tr[q - 1] = c * c;
    }
    tr[0] = Theta[j - 1] * Theta[j - 1];
    tr[k] = Theta[j] * Theta[j];
    for (int q = 1; q <= k; ++q)
      g->fracirg[(size_t)g->off[j - 1] + (q - 1)] =
          (cos(thet[j - 1] + (double)(float)(q - 1) * dth) - cos(thet[j - 1] + (double)(float)q * dth)) /
          (Theta[j - 1] - Theta[j]);
  }
}

/* the sub-cell of a point at polar angle theta (its |z|/r) in row j
 * (TraceMono.f:1631-1637, 1159-1164, 2269-2275) */
SF_HD int sf_irg(const SfGeom &g, const double *thet, int j, double theta) {
  const int k = g.nrg[j - 1];
  if (k <= 1 || !(theta == theta)) return 1;
  int irg = (int)((double)(float)k * (theta - thet[j - 1]) / (thet[j] - thet[j - 1])) + 1;
  if (irg > k) irg = k;
  if (irg < 1) irg = 1;
  return irg;
}

/* Trace2edgeRG, TraceMono.f:2487-2657.  Returns 1 when nothing can be hit
 * (the reference stops the program there). */
SF_HD int sf_trace2edge_rg(const TModel &m, const SfGeom &g, TPkt &p, int irg, double *v, int *inext, int *jnext,
                           int *irgnext) {
  const int nt = m.nt;
  const int nrg = g.nrg[p.j - 1];
  const double r = (p.x * p.x + p.y * p.y) + p.z * p.z;
  const double Ra = m.R[p.i], Rb = m.R[p.i + 1];
  const double R1 = Ra * Ra, R2 = Rb * Rb;
  double T1, T2;
  if (nrg <= 1) {
    T1 = m.Theta[p.j - 1] * m.Theta[p.j - 1];
    T2 = m.Theta[p.j] * m.Theta[p.j];
  } else {
    const double *tr = g.thetrg + g.off[p.j - 1] + (p.j - 1);
    T1 = tr[irg - 1];
    T2 = tr[irg];
  }
  const double b = 2.0 * ((p.x * p.vx + p.y * p.vy) + p.z * p.vz);
  int hR1, hR2, hT1, hT2;
  double vR1, vR2, vT1, vT2;
  const bool top = p.j != nt - 1 || irg != nrg, bottom = p.j != 1 || irg != 1;
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
    if (top) {
      hT2 = tp_hitT(p, T2, r, b, &vT2);
    } else {
      vT2 = -p.z / p.vz;
      hT2 = vT2 > 0.0;
    }
  } else {
    hR1 = tp_hitR(R1, r, b, &vR1);
    hR2 = tp_hitR(R2, r, b, &vR2);
    if (bottom) {
      hT1 = tp_hitT(p, T1, r, b, &vT1);
    } else {
      hT1 = 0;
      vT1 = 1e200;
    }
    if (top) {
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
  *irgnext = irg;
  if (hR1 && vR1 < *v) {
    *v = vR1;
    *inext = p.i - 1;
    *jnext = p.j;
    *irgnext = irg;
    p.edgeNr = 2;
  }
  if (hR2 && vR2 < *v) {
    *v = vR2;
    *inext = p.i + 1;
    *jnext = p.j;
    *irgnext = irg;
    p.edgeNr = 1;
  }
  if (hT1 && vT1 < *v) {
    *v = vT1;
    *inext = p.i;
    if (nrg > 1) {
      *irgnext = irg - 1;
      *jnext = p.j;
      if (*irgnext < 1) {
        *jnext = p.j - 1;
        *irgnext = *jnext > 0 ? g.nrg[*jnext - 1] : 1;
      }
    } else {
      *jnext = p.j - 1;
      if (*jnext > 0) *irgnext = g.nrg[*jnext - 1];
    }
    p.edgeNr = 4;
  }
  if (hT2 && vT2 < *v) {
    *v = vT2;
    *inext = p.i;
    if (nrg > 1) {
      *irgnext = irg + 1;
      *jnext = p.j;
      if (*irgnext > nrg) {
        *jnext = p.j + 1;
        *irgnext = 1;
        if (*jnext == nt) *irgnext = g.nrg[nt - 2];
      }
    } else {
      *jnext = p.j + 1;
      *irgnext = 1;
    }
    p.edgeNr = 3;
  }
  if (*jnext == nt) {
    *jnext = nt - 1;
    *irgnext = g.nrg[nt - 2];
    p.edgeNr = 4;
  }
  if (*jnext == 0) {
    *jnext = 1;
    *irgnext = 1;
    p.edgeNr = 3;
  }
  return 0;
}

/* the folded azimuth bin 1..90 of a path point (trace2dpath,
 * TraceMono.f:2378-2382): phi in degrees, negative below the x axis,
 * truncated to one of NPHISCATT bins and folded onto half a circle */
SF_HD int sf_jphi(double x, double y) {
  const double rho = sqrt(x * x + y * y); /* a point on the axis takes phi = 0 */
  double phi = rho > 0.0 ? (180.0 * acos(fmin(1.0, fmax(-1.0, x / rho)))) / TP_PI : 0.0;
  if (y < 0.0) phi = -phi;
  int j = (int)(((double)(float)SF_NPHI * phi) / 360.0);
  j = j + 1;
  if (j < 1) j = 1 - j;
  if (j > SF_NPHI / 2) j = SF_NPHI + 1 - j;
  return j;
}

/* wavelength bracket of TraceMono (TraceMono.f:617-643): lam0 at or below
 * the first grid point takes (1, 2) with weights (1, 0) */
SF_HD void sf_lam(int nlam, const double *lam, double lam0, int *l1, int *l2, double *w1, double *w2) {
  *l1 = 0;
  *l2 = 1;
  *w1 = 1.0;
  *w2 = 0.0;
  for (int i = 0; i < nlam - 1; ++i)
    if (lam0 >= lam[i] && lam0 <= lam[i + 1]) {
      *l1 = i;
      *l2 = i + 1;
      *w1 = (lam[i + 1] - lam0) / (lam[i + 1] - lam[i]);
      *w2 = (lam0 - lam[i]) / (lam[i + 1] - lam[i]);
    }
  if (lam0 >= lam[nlam - 1]) {
    *l1 = nlam - 2;
    *l2 = nlam - 1;
    *w1 = 0.0;
    *w2 = 1.0;
  }
}

/* the cell's opacities at the wavelength (TraceMono.f:695-705): Kabs, Kext
 * (component Kabs + Ksca), Ksca and the albedo */
SF_HD void sf_cell_opac(int c, int ncomp, int nlam, const double *comp_w, const double *Kabs_c, const double *Ksca_c,
                        int l1, int l2, double w1, double w2, double *kabs, double *kext, double *ksca,
                        double *albedo) {
  const double *w = comp_w + (size_t)c * ncomp;
  double Ka = 0.0, Ke = 0.0, Ks = 0.0;
  for (int q = 0; q < ncomp; ++q) {
    const double *a = Kabs_c + (size_t)q * nlam, *s = Ksca_c + (size_t)q * nlam;
    Ka = Ka + (w1 * a[l1] + w2 * a[l2]) * w[q];
    Ke = Ke + (w1 * (a[l1] + s[l1]) + w2 * (a[l2] + s[l2])) * w[q];
    Ks = Ks + (w1 * s[l1] + w2 * s[l2]) * w[q];
  }
  *kabs = Ka;
  *kext = Ke;
  *ksca = Ks;
  *albedo = Ks / Ke;
}

/* element e of the cell's mixed Mueller matrix at the wavelength
 * (TraceMono.f:706-746): e < 1080 the element F[e / 180](e % 180 + 1),
 * e = 1080, 1081 the normalisations IF11, IF12; each the Ksca-weighted
 * mean over the components, sum_q (F_q(l1) Ksca_q(l1) w1 + F_q(l2)
 * Ksca_q(l2) w2) w_q / Ksca.  A cell that does not scatter has F11 = 1 and
 * the rest 0. */
SF_HD double sf_cell_mueller(int c, int e, int ncomp, int nlam, const double *comp_w, const double *Ksca_c,
                             const double *F_c, const double *IF_c, int l1, int l2, double w1, double w2,
                             double ksca) {
  if (ksca == 0.0) return (e < 180) ? 1.0 : 0.0;
  const double *w = comp_w + (size_t)c * ncomp;
  double s = 0.0;
  for (int q = 0; q < ncomp; ++q) {
    const double *ks = Ksca_c + (size_t)q * nlam;
    double f1, f2;
    if (e < 1080) {
      f1 = F_c[((size_t)q * nlam + l1) * 1080 + e];
      f2 = F_c[((size_t)q * nlam + l2) * 1080 + e];
    } else {
      f1 = IF_c[((size_t)q * nlam + l1) * 2 + (e - 1080)];
      f2 = IF_c[((size_t)q * nlam + l2) * 2 + (e - 1080)];
    }
    s = s + ((f1 * ks[l1]) * w1 + (f2 * ks[l2]) * w2) * w[q];
  }
  return s / ksca;
}

/* EmissionDistribution's thermal emission weight of a cell, thermal contact
 * (TraceMono.f:1029-1057): sum_q (w1 B(l1, T) Kabs_q(l1) + w2 B(l2, T)
 * Kabs_q(l2)) w_q, B linear between the 1 K points, times dens V */
SF_HD double sf_cell_emission(int c, int ncomp, int nlam, const double *comp_w, const double *Kabs_c, const double *BB,
                              double T, double dens, double V, int l1, int l2, double w1, double w2) {
  if (T == 0.0) return 0.0;
  int iT = (int)(T / 1.0);
  const double wT1 = (double)(iT + 1) - T / 1.0, wT2 = T / 1.0 - (double)iT;
  if (iT < 1) iT = 1;
  if (iT > TP_TMAX - 1) iT = TP_TMAX - 1;
  const double *B1 = BB + (size_t)l1 * TP_TT, *B2 = BB + (size_t)l2 * TP_TT;
  const double *w = comp_w + (size_t)c * ncomp;
  double e = 0.0;
  for (int q = 0; q < ncomp; ++q) {
    const double *a = Kabs_c + (size_t)q * nlam;
    e = e + ((w1 * (wT1 * B1[iT] + wT2 * B1[iT + 1])) * a[l1] + (w2 * (wT1 * B2[iT] + wT2 * B2[iT + 1])) * a[l2]) *
                w[q];
  }
  return (e * dens) * V;
}

/* the shortest absorption depth from the cell's centre to the outside over
 * nexits directions in the plane x = 0 (TraceMono.f:1076-1099, trace2exit
 * with withscatt false); kabs per cell.  Rays ended by a geometry failure
 * or the step cap count as reaching the outside with the depth so far. */
SF_HD double sf_tauexit(const TModel &m, const double *kabs, int i, int j, int nexits) {
  double taumin = 0.0;
  for (int k = 1; k <= nexits; ++k) {
    TPkt p;
    double Rad = 0.5;
    Rad = sqrt(m.R[i] * m.R[i] * Rad + m.R[i + 1] * m.R[i + 1] * (1.0 - Rad));
    double Th = 0.5;
    Th = m.Theta[j - 1] * Th + m.Theta[j] * (1.0 - Th);
    p.z = Rad * Th;
    double phi = 1e-4;
    p.x = Rad * sqrt(1.0 - Th * Th) * dm_sin(phi);
    p.y = Rad * sqrt(1.0 - Th * Th) * dm_cos(phi);
    phi = (TP_PI * (double)(float)(k - 1)) / (double)(float)(nexits - 1);
    p.vx = 0.0;
    p.vy = dm_cos(phi);
    p.vz = dm_sin(phi);
    p.i = i;
    p.j = j;
    p.onEdge = 0;
    p.edgeNr = 0;
    const int nc = m.nt - 1;
    double tau = 0.0;
    for (int n = 0; n < 1000000; ++n) {
      double v;
      int inext, jnext;
      if (tp_trace2edge(m, p, &v, &inext, &jnext) != 0) break;
      p.onEdge = 1;
      p.x = p.x + p.vx * v;
      p.y = p.y + p.vy * v;
      p.z = p.z + p.vz * v;
      const size_t c = (size_t)p.i * nc + (p.j - 1);
      tau = tau + ((v * m.dens[c]) * TP_AU) * kabs[c];
      if (inext >= m.nr || inext <= 0) break;
      p.i = inext;
      p.j = jnext;
    }
    if (tau < taumin || k == 1) taumin = tau;
  }
  return taumin;
}

/* the scattered source term of one path segment (TraceFlux,
 * TraceMono.f:356-395): the mean over the segment's folded azimuth bins
 * jphi1..jphi2 of albedo / (V fracirg) SF(bin) on the side the segment
 * ends on */
SF_HD double sf_segment_source(const SfGeom &g, const double *SF, int i, int j, int irg, int side, int jphi1,
                               int jphi2, double albedo, double V) {
  const size_t base = (((size_t)i * g.nsub + g.off[j - 1] + (irg - 1)) * 2 + side) * SF_NB;
  const double ww = albedo / (V * g.fracirg[g.off[j - 1] + (irg - 1)]);
  const int djj = jphi1 <= jphi2 ? 1 : -1;
  double x = 0.0;
  int n = 0;
  for (int jj = jphi1;; jj += djj) {
    x = x + ww * SF[base + jj];
    ++n;
    if (jj == jphi2) break;
  }
  return x / (double)(float)n;
}

#endif /* MCMAX_SCAT_CORE_CUH */
