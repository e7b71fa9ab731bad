/*
 * oracle_mc.c -- serial CPU restatement of MCMax's photon-packet loop.
 * Test infrastructure only (parity reference for the GPU transport kernels and the
 * timed CPU baseline).
 *
 * Follows:
 *   MCRadiation  MCRadiation.f:6-887   (star emission :355-382, packet loop
 *                                       :320-648, SED binning :576-646)
 *   trace2d      MCRadiation.f:901-1141
 *   Trace2edge   MCRadiation.f:1150-1272, hitR :1274, hitT :1306, hitTsame :1340
 *   interact     Radiation.f:41-355 (thermal-contact branch)
 *   scatangle    Radiation.f:381-495, RotateStokes :506-534
 *   emit         Radiation.f:940-1001, randomdirection :1007-1024
 *   rotate       Subroutines.f:1648-1675, hunt :2086-2132
 *   MinDist, RandomWalk  RandomWalk.f:15-147
 *
 * Differences from the reference, all deliberate and shared with the GPU
 * kernels:
 *   - opacities at the packet wavelength come from the per-cell totals
 *     KabsTot/KscaTot (the reference builds them in MCRadiation.f:199-236 and
 *     uses them in interact; trace2d re-sums the grains, which only differs by
 *     floating-point reassociation);
 *   - the Planck-mean table of a cell is the pre-summed KpCell[iT] and the
 *     re-emission normalisation kp is formed from it (linear in the grains);
 *   - random numbers: Philox4x32-10 per packet (rng = 0) or the reference's
 *     ran1 (rng = 1);
 *   - sin/cos/log come from detmath.h so the FP64 GPU path can replay a run
 *     bit for bit;
 *   - a packet whose cell search at emission finds no cell (|z|/R* exactly on
 *     a cone) takes the cell below; a zero-width emission interval takes its
 *     lower edge; an escape with |vz| = 1 goes to the last angle bin (the
 *     reference would index bin 31).
 * Options not built (not used by the hot-path configurations): per-grain
 * temperatures (tcontact = .false.), QHP grains, viscous / inner-gas / ISRF
 * emission, forced first interaction, multi-wavelength spectra, local
 * radiation field, radiation pressure, etrace.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "../mcmax_b200/csrc/detmath.h"
#include "../mcmax_b200/csrc/philox.h"

/* AU as the reference holds it: a single-precision literal widened to
 * real*8 (Modules.f:4,8) */
#define AU_CM ((double)1.49598e13f)
#define PI_D 3.14159265358979323846
#define NY_RW 1000

typedef struct {
  double x, y, z, vx, vy, vz, E, Q, U, V, Sx, Sy, Sz;
  double wl1, wl2;
  int ilam1, ilam2, edgeNr, i, j;
  int onEdge, scatt, pol;
} orc_phot;

typedef struct {
  int rng;
  px_stream px;
  int32_t idum, iv[32], iy;
} rng_t;

static double rnd(rng_t *r) {
  if (r->rng == 0) return px_next(&r->px);
  return orc_ran1(&r->idum, r->iv, &r->iy);
}

typedef struct {
  const orc_model *m;
  orc_result *out;
  int nc;         /* theta cells per radius = nt-1 */
  int scattering; /* any Ksca > 0 and scat_how != 0 */
  int scat_how;
  int rw;
  double factRW;
  double *mass;
  double *Tcell;
  int *lastphot;
  int *iTD;
  double *kdext, *kdabs;
  double nEJv;
} mc_t;

static inline int cidx(const mc_t *s, int i, int j) { return i * s->nc + (j - 1); }

static void randomdirection(rng_t *r, double *x, double *y, double *z) {
  double rr;
  for (;;) {
    *x = 2.0 * rnd(r) - 1.0;
    *y = 2.0 * rnd(r) - 1.0;
    *z = 2.0 * rnd(r) - 1.0;
    rr = ((*x) * (*x) + (*y) * (*y)) + (*z) * (*z);
    if (!(rr > 1.0)) break;
  }
  rr = sqrt(rr);
  *x = *x / rr;
  *y = *y / rr;
  *z = *z / rr;
}

static void set_s_from_v(orc_phot *p) {
  double x = -p->vy, y = p->vx, z = 0.0;
  double r = sqrt((x * x + y * y) + z * z);
  p->Sx = x / r;
  p->Sy = y / r;
  p->Sz = z / r;
}

/* emit from a spectrum given as a callback-free array (Radiation.f:940-1001) */
static void emit_scan(mc_t *s, rng_t *r, orc_phot *p, const double *spec, double Lttot) {
  const orc_model *m = s->m;
  s->out->counters[0]++;
  randomdirection(r, &p->vx, &p->vy, &p->vz);
  p->scatt = 0;
  p->pol = 0;
  set_s_from_v(p);
  double Lr = rnd(r) * Lttot;
  double Ltold = 0.0, Lt = 0.0;
  for (int i = 0; i < m->nlam - 1; ++i) {
    Lt = Lt + (fabs(m->nu[i] - m->nu[i + 1]) * 0.5) * (spec[i] + spec[i + 1]);
    if (Lt >= Lr) {
      double d = Lt - Ltold;
      p->wl1 = d != 0.0 ? (Lr - Ltold) / d : 1.0;
      p->wl2 = 1.0 - p->wl1;
      p->ilam1 = i;
      p->ilam2 = i + 1;
      return;
    }
    Ltold = Lt;
  }
  p->wl1 = 0.0;
  p->wl2 = 1.0;
  p->ilam1 = m->nlam - 2;
  p->ilam2 = m->nlam - 1;
}

static int hitR(double Rad, double r, double b, double *v) {
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

static int hitT(const orc_phot *p, double Thet, double r, double b, double *v) {
  int hit = 0;
  *v = 1e200;
  double at = Thet - p->vz * p->vz;
  double bt = Thet * b - (2.0 * p->z) * p->vz;
  double ct = Thet * r - p->z * p->z;
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

static int hitTsame(const orc_phot *p, double Thet, double b, double *v) {
  double bt = Thet * b - (2.0 * p->z) * p->vz;
  double at = Thet - p->vz * p->vz;
  *v = (-bt) / at;
  return *v > 0.0;
}

/* returns 0 on success, 1 when nothing can be hit (reference: stop) */
static int trace2edge(mc_t *s, orc_phot *p, double *v, int *inext, int *jnext) {
  const orc_model *m = s->m;
  int nt = m->nt;
  double r = (p->x * p->x + p->y * p->y) + p->z * p->z;
  double R1 = m->R[p->i] * m->R[p->i];
  double R2 = m->R[p->i + 1] * m->R[p->i + 1];
  double T1 = m->Theta[p->j - 1] * m->Theta[p->j - 1];
  double T2 = m->Theta[p->j] * m->Theta[p->j];
  double b = 2.0 * ((p->x * p->vx + p->y * p->vy) + p->z * p->vz);
  int hR1, hR2, hT1, hT2;
  double vR1, vR2, vT1, vT2;
  if (!p->onEdge) {
    hR1 = hitR(R1, r, b, &vR1);
    hR2 = hitR(R2, r, b, &vR2);
    hT1 = hitT(p, T1, r, b, &vT1);
    hT2 = hitT(p, T2, r, b, &vT2);
  } else if (p->edgeNr == 1) {
    hR1 = 0;
    vR1 = 1e200;
    hR2 = hitR(R2, r, b, &vR2);
    hT1 = hitT(p, T1, r, b, &vT1);
    hT2 = hitT(p, T2, r, b, &vT2);
  } else if (p->edgeNr == 2) {
    hR1 = hitR(R1, r, b, &vR1);
    hR2 = 1;
    vR2 = -b;
    hT1 = hitT(p, T1, r, b, &vT1);
    hT2 = hitT(p, T2, r, b, &vT2);
  } else if (p->edgeNr == 3) {
    hR1 = hitR(R1, r, b, &vR1);
    hR2 = hitR(R2, r, b, &vR2);
    hT1 = 0;
    vT1 = 1e200;
    if (p->j != nt - 1) {
      hT2 = hitT(p, T2, r, b, &vT2);
    } else {
      vT2 = -p->z / p->vz;
      hT2 = vT2 > 0.0;
    }
  } else {
    hR1 = hitR(R1, r, b, &vR1);
    hR2 = hitR(R2, r, b, &vR2);
    if (p->j != 1) {
      hT1 = hitT(p, T1, r, b, &vT1);
    } else {
      hT1 = 0;
      vT1 = 1e200;
    }
    if (p->j != nt - 1) {
      hT2 = hitTsame(p, T2, b, &vT2);
    } else {
      hT2 = 0;
      vT2 = 1e200;
    }
  }
  if (!hR1 && !hR2 && !hT1 && !hT2) {
    hR1 = hitR(R1, r, b, &vR1);
    hR2 = hitR(R2, r, b, &vR2);
    hT1 = hitT(p, T1, r, b, &vT1);
    hT2 = hitT(p, T2, r, b, &vT2);
    if (!hR1 && !hR2 && !hT1 && !hT2) return 1;
  }
  *v = 1e200;
  *inext = p->i;
  *jnext = p->j;
  if (hR1 && vR1 < *v) {
    *v = vR1;
    *inext = p->i - 1;
    *jnext = p->j;
    p->edgeNr = 2;
  }
  if (hR2 && vR2 < *v) {
    *v = vR2;
    *inext = p->i + 1;
    *jnext = p->j;
    p->edgeNr = 1;
  }
  if (hT1 && vT1 < *v) {
    *v = vT1;
    *inext = p->i;
    *jnext = p->j - 1;
    p->edgeNr = 4;
  }
  if (hT2 && vT2 < *v) {
    *v = vT2;
    *inext = p->i;
    *jnext = p->j + 1;
    p->edgeNr = 3;
  }
  if (*jnext == nt) {
    *jnext = nt - 1;
    p->edgeNr = 4;
  }
  if (*jnext == 0) {
    *jnext = 1;
    p->edgeNr = 3;
  }
  return 0;
}

static void rotate(double *x, double *y, double *z, double u, double v, double w, double theta) {
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

static void rotate_stokes(orc_phot *p, double x, double y, double z) {
  double P = (p->U / p->E) * (p->U / p->E) + (p->Q / p->E) * (p->Q / p->E);
  if (P == 0.0) return;
  double cost = (p->Sx * x + p->Sy * y) + p->Sz * z;
  double sint = (x - (p->Sx * (p->vy * p->vy + p->vz * p->vz) - p->vx * (p->vy * p->Sy + p->vz * p->Sz)) * cost) /
                (p->vy * p->Sz - p->vz * p->Sy);
  double cos2t = cost * cost - sint * sint;
  double sin2t = (2.0 * sint) * cost;
  double Q = p->Q * cos2t + p->U * sin2t;
  double U = (-p->Q) * sin2t + p->U * cos2t;
  double P2 = (U / p->E) * (U / p->E) + (Q / p->E) * (Q / p->E);
  double sPP2 = sqrt(P / P2);
  p->U = sPP2 * U;
  p->Q = sPP2 * Q;
}

/* Radiation.f:381-495 for the component matrix F[6*180] and IF[2] */
static void scatangle(mc_t *s, rng_t *r, orc_phot *p, const double *F, const double *IF) {
  const orc_model *m = s->m;
  const double *F11 = F, *F12 = F + 180, *F22 = F + 360, *F33 = F + 540, *F34 = F + 720, *F44 = F + 900;
  double IF11 = IF[0] * 180.0, IF12 = IF[1] * 180.0;
  double phi;
  if (p->pol) {
    double Itot = 0.0;
    for (int i = 1; i <= 180; ++i)
      Itot = (Itot + IF11 * p->E) + IF12 * (p->Q * m->cos2phi[i] + p->U * m->sin2phi[i]);
    Itot = rnd(r) * Itot;
    double I1 = 0.0, I0 = 0.0;
    phi = PI_D;
    for (int i = 1; i <= 180; ++i) {
      I0 = (I0 + IF11 * p->E) + IF12 * (p->Q * m->cos2phi[i] + p->U * m->sin2phi[i]);
      if (I0 > Itot) {
        double wp1 = (I0 - Itot) / (I0 - I1);
        phi = (PI_D * ((double)i - wp1)) / 180.0;
        break;
      }
      I1 = I0;
    }
  } else {
    phi = rnd(r) * PI_D;
  }
  double x = p->Sx, y = p->Sy, z = p->Sz;
  rotate(&x, &y, &z, p->vx, p->vy, p->vz, phi);
  if (p->pol) rotate_stokes(p, x, y, z);
  p->Sx = x;
  p->Sy = y;
  p->Sz = z;
  double Fr = 180.0 * (p->E * IF[0] + p->Q * IF[1]);
  Fr = rnd(r) * Fr;
  double Fi = 0.0, FiOld = 0.0, theta = PI_D;
  int ib = 180;
  for (int i = 1; i <= 180; ++i) {
    Fi = Fi + (PI_D * m->sinthet[i - 1]) * (F11[i - 1] * p->E + F12[i - 1] * p->Q);
    if (Fi > Fr) {
      theta = (double)i - (Fi - Fr) / (Fi - FiOld);
      theta = (theta * PI_D) / 180.0;
      ib = i;
      break;
    }
    FiOld = Fi;
  }
  if (rnd(r) < 0.5) theta = -theta;
  int k = ib - 1;
  double E = (0.0 + F11[k] * p->E) + F12[k] * p->Q;
  double Q = (0.0 + F12[k] * p->E) + F22[k] * p->Q;
  double U = 0.0 + F33[k] * p->U;
  double Fs = (theta >= 0.0 && !signbit(theta)) ? fabs(F34[k]) : -fabs(F34[k]);
  U = U + Fs * p->V;
  double V = (0.0 - Fs * p->U) + F44[k] * p->V;
  if (E != 0.0) {
    p->Q = (p->E * Q) / E;
    p->U = (p->E * U) / E;
    p->V = (p->E * V) / E;
  }
  rotate(&p->vx, &p->vy, &p->vz, p->Sx, p->Sy, p->Sz, theta);
  double rr = sqrt((p->vx * p->vx + p->vy * p->vy) + p->vz * p->vz);
  p->vx /= rr;
  p->vy /= rr;
  p->vz /= rr;
  rr = sqrt((p->Sx * p->Sx + p->Sy * p->Sy) + p->Sz * p->Sz);
  p->Sx /= rr;
  p->Sy /= rr;
  p->Sz /= rr;
  if (ib != 1 && ib != 180) p->pol = 1;
}

/* interact, thermal-contact branch (Radiation.f:41-76, :160-258, :262-315) */
static void interact(mc_t *s, rng_t *r, orc_phot *p) {
  const orc_model *m = s->m;
  int c = cidx(s, p->i, p->j);
  int nlam = m->nlam;
  const double *KabsT = m->KabsTot + (size_t)c * nlam;
  const double *KscaT = m->KscaTot + (size_t)c * nlam;
  double Ksca = KscaT[p->ilam1] * p->wl1 + KscaT[p->ilam2] * p->wl2;
  double Kext = Ksca + (KabsT[p->ilam1] * p->wl1 + KabsT[p->ilam2] * p->wl2);
  double KabsTot = Kext - Ksca;
  double Albedo = Ksca / Kext;
  s->out->counters[1]++;
  if (!s->scattering || rnd(r) > Albedo) {
    s->out->counters[2]++;
    if (s->out->Nabs) s->out->Nabs[c] += 1;
    p->scatt = 0;
    p->pol = 0;
    p->Q = 0.0;
    p->U = 0.0;
    p->V = 0.0;
    const double *kp = m->KpCell + (m->kp_uniform ? (size_t)0 : (size_t)c * (ORC_TMAX + 1));
    s->out->Eabs[c] = s->out->Eabs[c] + (p->E * (KabsTot - 0.0)) / KabsTot;
    double T0 = s->Tcell[c];
    double T1 = orc_increase_t(kp, s->out->Eabs[c] / s->mass[c], T0);
    int iT0 = (int)(T0 / 1.0), iT1 = (int)(T1 / 1.0);
    double epsT0 = T0 - (double)iT0 * 1.0, epsT1 = T1 - (double)iT1 * 1.0;
    if (iT0 >= ORC_TMAX - 1) iT0 = ORC_TMAX - 2;
    if (iT1 >= ORC_TMAX - 1) iT1 = ORC_TMAX - 1;
    if (iT0 < 1) iT0 = 1;
    if (iT1 < 2) iT1 = 2;
    double *spec = (double *)malloc(sizeof(double) * (size_t)nlam);
    const int TT = ORC_TMAX + 1;
    double kpe;
    if (iT0 == iT1) {
      for (int l = 0; l < nlam; ++l)
        spec[l] = (m->BB[(size_t)l * TT + iT0 + 1] - m->BB[(size_t)l * TT + iT0]) * KabsT[l];
      kpe = kp[iT0 + 1] - kp[iT0];
    } else {
      for (int l = 0; l < nlam; ++l) {
        const double *B = m->BB + (size_t)l * TT;
        spec[l] = (((epsT1 * B[iT1 + 1] + (1.0 - epsT1) * B[iT1]) - epsT0 * B[iT0 + 1]) - (1.0 - epsT0) * B[iT0]) * KabsT[l];
      }
      kpe = ((epsT1 * kp[iT1 + 1] + (1.0 - epsT1) * kp[iT1]) - epsT0 * kp[iT0 + 1]) - (1.0 - epsT0) * kp[iT0];
    }
    if (kpe == 0.0) {
      for (int l = 0; l < nlam; ++l) spec[l] = 0.0;
      kpe = 0.0 / KabsTot;
    }
    emit_scan(s, r, p, spec, kpe);
    free(spec);
    s->Tcell[c] = T1;
  } else {
    s->out->counters[3]++;
    p->scatt = 1;
    if (s->scat_how == 1) {
      randomdirection(r, &p->vx, &p->vy, &p->vz);
    } else {
      double KscaR = Ksca * rnd(r);
      const double *F = NULL, *IF = NULL;
      for (int q = 0; q < m->ncomp && F == NULL; ++q) {
        double w1 = m->comp_w[(size_t)c * m->ncomp + q];
        double w2 = (w1 * p->wl2) * m->Ksca_comp[(size_t)q * nlam + p->ilam2];
        KscaR = KscaR - w2;
        if (KscaR < 0.0) {
          F = m->F_comp + ((size_t)q * nlam + p->ilam2) * 1080;
          IF = m->IF_comp + ((size_t)q * nlam + p->ilam2) * 2;
          break;
        }
        w1 = (w1 * p->wl1) * m->Ksca_comp[(size_t)q * nlam + p->ilam1];
        KscaR = KscaR - w1;
        if (KscaR < 0.0) {
          F = m->F_comp + ((size_t)q * nlam + p->ilam1) * 1080;
          IF = m->IF_comp + ((size_t)q * nlam + p->ilam1) * 2;
          break;
        }
      }
      double Mavg[1080], IFavg[2];
      if (F == NULL) {
        /* averaged matrix fallback, Radiation.f:293-315 */
        memset(Mavg, 0, sizeof Mavg);
        IFavg[0] = IFavg[1] = 0.0;
        for (int q = 0; q < m->ncomp; ++q) {
          double w1 = m->comp_w[(size_t)c * m->ncomp + q];
          double w2 = ((w1 * p->wl2) * m->Ksca_comp[(size_t)q * nlam + p->ilam2]) / Ksca;
          w1 = ((w1 * p->wl1) * m->Ksca_comp[(size_t)q * nlam + p->ilam1]) / Ksca;
          const double *Fa = m->F_comp + ((size_t)q * nlam + p->ilam1) * 1080;
          const double *Fb = m->F_comp + ((size_t)q * nlam + p->ilam2) * 1080;
          const double *Ia = m->IF_comp + ((size_t)q * nlam + p->ilam1) * 2;
          const double *Ib = m->IF_comp + ((size_t)q * nlam + p->ilam2) * 2;
          IFavg[0] = (IFavg[0] + w1 * Ia[0]) + w2 * Ib[0];
          IFavg[1] = (IFavg[1] + w1 * Ia[1]) + w2 * Ib[1];
          for (int e = 0; e < 1080; ++e) Mavg[e] = (Mavg[e] + w1 * Fa[e]) + w2 * Fb[e];
        }
        F = Mavg;
        IF = IFavg;
        s->out->counters[10]++;
      }
      scatangle(s, r, p, F, IF);
    }
  }
}

static double mindist(mc_t *s, const orc_phot *p) {
  const orc_model *m = s->m;
  double rho = p->x * p->x + p->y * p->y;
  double r = sqrt(rho + p->z * p->z);
  rho = sqrt(rho);
  double z = fabs(p->z);
  double R1 = m->R[p->i], R2 = m->R[p->i + 1];
  double T1 = m->Theta[p->j - 1], T2 = m->Theta[p->j];
  double ST1 = m->SinTheta[p->j - 1], ST2 = m->SinTheta[p->j];
  double vR1 = fabs(r - R1), vR2 = fabs(R2 - r);
  double vT1 = fabs(T1 * rho - ST1 * z), vT2 = fabs(T2 * rho - ST2 * z);
  double d = vR1;
  if (vR2 < d) d = vR2;
  if (vT1 < d) d = vT1;
  if (vT2 < d) d = vT2;
  return d;
}

/* Numerical Recipes hunt on a table of n entries, 1-based jlo in/out */
static void hunt(const double *xx, int n, double x, int *jlo) {
  int jhi, jm, inc;
  int ascnd = xx[n - 1] >= xx[0];
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

/* DiffCoeffCell (Dtable.f:97-182) for one cell and one iT */
static void orc_diffcoeff_one(const orc_model *m, int c, int iT, int scattering, double *kdext, double *kdabs) {
  const int nlam = m->nlam, TT = ORC_TMAX + 1;
  const double *Ka = m->KabsTot + (size_t)c * nlam, *Ks = m->KscaTot + (size_t)c * nlam;
  const double *w = m->comp_w + (size_t)c * m->ncomp;
  double int1 = 0.0, int2 = 0.0, int3 = 0.0, b0 = 0.0, e0 = 0.0, a0 = 0.0;
  for (int l = 0; l < nlam; ++l) {
    double g = 0.0;
    for (int q = 0; q < m->ncomp; ++q) g = g + (m->g_comp[(size_t)q * nlam + l] * m->Ksca_comp[(size_t)q * nlam + l]) * w[q];
    g = g / Ks[l];
    if (!scattering) g = 0.0;
    double Kext = Ka[l] + Ks[l];
    double b1 = m->BB[(size_t)l * TT + iT + 1] - m->BB[(size_t)l * TT + iT];
    double e1 = b1 / (Kext - (g * g) * Ks[l]), a1 = b1 * (Ka[l] - 0.0);
    if (l > 0) {
      double dh = fabs(m->nu[l - 1] - m->nu[l]) * 0.5;
      int1 = int1 + dh * (e0 + e1);
      int2 = int2 + dh * (b0 + b1);
      int3 = int3 + dh * (a0 + a1);
    }
    b0 = b1;
    e0 = e1;
    a0 = a1;
  }
  *kdext = int2 / int1;
  *kdabs = int3 / int2;
}

/* RandomWalk.f:47-147 (thermal contact); returns 1 when a step was taken */
static int random_walk(mc_t *s, rng_t *r, orc_phot *p, double dmin) {
  const orc_model *m = s->m;
  int c = cidx(s, p->i, p->j);
  int iT = (int)(s->Tcell[c] / 1.0);
  if (iT == 0) iT = 1;
  if (iT > ORC_TMAX) iT = ORC_TMAX;
  if (iT > ORC_TMAX - 1) iT = ORC_TMAX - 1; /* DiffCoeffCell clamp */
  double Kext, KabsD;
  if (m->KDext) {
    Kext = m->KDext[(size_t)c * (ORC_TMAX + 1) + iT];
    KabsD = m->KDabs[(size_t)c * (ORC_TMAX + 1) + iT];
  } else {
    /* DiffCoeffCell only when the cell's temperature step changed
     * (RandomWalk.f:61, Dtable.f:97-182) */
    if (s->iTD[c] != iT) {
      orc_diffcoeff_one(m, c, iT, s->scattering, &s->kdext[c], &s->kdabs[c]);
      s->iTD[c] = iT;
    }
    Kext = s->kdext[c];
    KabsD = s->kdabs[c];
  }
  double lr = 1.0 / ((AU_CM * Kext) * m->dens[c]);
  if (dmin <= s->factRW * lr) return 0;
  double x = rnd(r);
  int iy = 1;
  hunt(m->rw_phi, NY_RW, x, &iy);
  double v = (((-3.0 * dm_log(m->rw_y[iy - 1])) * (dmin * dmin)) / (lr * (PI_D * PI_D)));
  double Kabs = KabsD;
  randomdirection(r, &p->vx, &p->vy, &p->vz);
  p->x = p->x + dmin * p->vx;
  p->y = p->y + dmin * p->vy;
  p->z = p->z + dmin * p->vz;
  double EJv = (p->E * v) * AU_CM;
  s->out->Eabs[c] = s->out->Eabs[c] + (EJv * Kabs) * m->dens[c];
  s->out->EJv[c] = s->out->EJv[c] + EJv * Kabs;
  s->nEJv = s->nEJv + EJv * Kabs;
  const double *kp = m->KpCell + (m->kp_uniform ? (size_t)0 : (size_t)c * (ORC_TMAX + 1));
  s->Tcell[c] = orc_increase_t(kp, s->out->Eabs[c] / s->mass[c], s->Tcell[c]);
  s->out->tautot += v / dmin;
  s->out->counters[4]++;
  return 1;
}

/* trace2d, MCRadiation.f:901-1141.  Returns 0 interaction, 1 escape, 2 star
 * hit / abandoned, -1 geometry failure. */
static int trace2d(mc_t *s, rng_t *r, orc_phot *p, double tau0, int64_t pid) {
  const orc_model *m = s->m;
  int nlam = m->nlam;
  double tau = 0.0;
  int ntrace = 0;
  if (s->rw && m->thick && m->thick[cidx(s, p->i, p->j)] && !p->onEdge) {
    for (;;) {
      double dmin = mindist(s, p);
      if (!random_walk(s, r, p, dmin)) break;
      double vx, vy, vz, inp;
      do {
        randomdirection(r, &vx, &vy, &vz);
        inp = (p->vx * vx + p->vy * vy) + p->vz * vz;
      } while (inp < 0.0);
      p->vx = vx;
      p->vy = vy;
      p->vz = vz;
    }
  }
  for (;;) {
    int c = cidx(s, p->i, p->j);
    if (s->lastphot[c] != (int)(pid + 1)) {
      s->out->Ni[c] += 1;
      s->lastphot[c] = (int)(pid + 1);
    }
    const double *KabsT = m->KabsTot + (size_t)c * nlam;
    const double *KscaT = m->KscaTot + (size_t)c * nlam;
    double Kabs = KabsT[p->ilam1] * p->wl1 + KabsT[p->ilam2] * p->wl2;
    double Kext = Kabs;
    if (s->scattering) Kext = (KscaT[p->ilam1] * p->wl1 + KscaT[p->ilam2] * p->wl2) + Kabs;
    double KabsBB = Kabs;
    double v;
    int inext, jnext;
    if (trace2edge(s, p, &v, &inext, &jnext)) return -1;
    s->out->counters[8]++;
    double tau1 = ((Kext * v) * m->dens[c]) * AU_CM;
    if (tau + tau1 > tau0) {
      v = (v * (tau0 - tau)) / tau1;
      tau1 = tau0 - tau;
      s->out->tautot += tau1;
      p->x = p->x + p->vx * v;
      p->y = p->y + p->vy * v;
      p->z = p->z + p->vz * v;
      p->onEdge = 0;
      double EJv = (p->E * v) * AU_CM;
      s->out->EJv[c] = s->out->EJv[c] + EJv * KabsBB;
      s->nEJv = s->nEJv + EJv * KabsBB;
      return 0;
    }
    p->x = p->x + p->vx * v;
    p->y = p->y + p->vy * v;
    p->z = p->z + p->vz * v;
    double EJv = (p->E * v) * AU_CM;
    s->nEJv = s->nEJv + EJv * KabsBB;
    s->out->EJv2[c] = s->out->EJv2[c] + s->nEJv * s->nEJv;
    s->nEJv = 0.0;
    s->out->EJv[c] = s->out->EJv[c] + EJv * KabsBB;
    p->onEdge = 1;
    tau = tau + tau1;
    s->out->tautot += tau1;
    if (inext >= m->nr) return 1;
    if (inext < 0) return 2;
    p->i = inext;
    p->j = jnext;
    ntrace++;
    if (tau < 0.0) return 2;
    if (ntrace > m->nr * m->nt * 2) {
      s->out->counters[6]++;
      return 2;
    }
  }
}

int orc_mcradiation(const orc_model *m, const orc_run *run, orc_result *out) {
  const int nr = m->nr, nt = m->nt, nlam = m->nlam;
  const int nc = nt - 1;
  const int ncell = nr * nc;
  mc_t S;
  memset(&S, 0, sizeof S);
  S.m = m;
  S.out = out;
  S.nc = nc;
  S.scat_how = run->scat_how;
  S.scattering = 0;
  if (run->scat_how != 0)
    for (size_t k = 0; k < (size_t)ncell * nlam; ++k)
      if (m->KscaTot[k] != 0.0) {
        S.scattering = 1;
        break;
      }
  S.rw = run->randomwalk;
  S.factRW = run->factRW;
  S.mass = (double *)malloc(sizeof(double) * ncell);
  S.Tcell = (double *)calloc(ncell, sizeof(double));
  S.lastphot = (int *)calloc(ncell, sizeof(int));
  S.iTD = (int *)calloc(ncell, sizeof(int));
  S.kdext = (double *)calloc(ncell, sizeof(double));
  S.kdabs = (double *)calloc(ncell, sizeof(double));
  for (int c = 0; c < ncell; ++c) S.mass[c] = m->dens[c] * m->V[c];
  /* the transport floors the dust density at 1e-50 (CheckMinimumDensity,
   * DiskStructure.f:2966-2979) after the mass was formed */
  double *dens = (double *)malloc(sizeof(double) * ncell);
  for (int c = 0; c < ncell; ++c) dens[c] = m->dens[c] <= 1e-50 ? 1e-50 : m->dens[c];
  orc_model mm = *m;
  mm.dens = dens;
  S.m = &mm;

  memset(out->EJv, 0, sizeof(double) * ncell);
  memset(out->EJv2, 0, sizeof(double) * ncell);
  memset(out->Eabs, 0, sizeof(double) * ncell);
  memset(out->Ni, 0, sizeof(int32_t) * ncell);
  if (out->Nabs) memset(out->Nabs, 0, sizeof(int32_t) * ncell);
  memset(out->spec, 0, sizeof(double) * nlam * (ORC_NANGLE_SED + 1));
  memset(out->scatspec, 0, sizeof(double) * nlam * (ORC_NANGLE_SED + 1));
  memset(out->ispec, 0, sizeof(int32_t) * nlam * (ORC_NANGLE_SED + 1));
  memset(out->counters, 0, sizeof out->counters);
  out->tautot = 0.0;

  /* SED weights, MCRadiation.f:52-80 */
  double *wlam = (double *)malloc(sizeof(double) * nlam);
  for (int i = 0; i < nlam; ++i) {
    if (i == 0)
      wlam[i] = -1e23 / (m->nu[1] / 2.0);
    else if (i == nlam - 1)
      wlam[i] = -1e23 / ((m->nu[nlam - 1] - m->nu[nlam - 2]) / 2.0);
    else
      wlam[i] = -1e23 / ((m->nu[i + 1] - m->nu[i - 1]) / 2.0);
  }
  double wangle[ORC_NANGLE_SED + 1];
  for (int i = 1; i <= ORC_NANGLE_SED; ++i)
    wangle[i] = 1.0 / ((double)i / (double)ORC_NANGLE_SED - (double)(i - 1) / (double)ORC_NANGLE_SED);

  rng_t R;
  memset(&R, 0, sizeof R);
  R.rng = run->rng;
  R.idum = run->idum;
  const int64_t Nphot = run->nphot;
  const double Epkt = m->Lstar / ((double)Nphot * 1.0);
  int status = 0;

  for (int64_t ip = 0; ip < Nphot; ++ip) {
    if (R.rng == 0) px_init(&R.px, run->seed, (uint64_t)ip);
    orc_phot p;
    memset(&p, 0, sizeof p);
    int done = 0;
    while (!done) {
      /* (re-)emission from the star, MCRadiation.f:350-382 */
      S.nEJv = 0.0;
      int64_t ninteract = 0;
      (void)rnd(&R); /* where_emit */
      double x, y, z;
      randomdirection(&R, &x, &y, &z);
      p.x = m->R[0] * x;
      p.y = m->R[0] * y;
      p.z = m->R[0] * z;
      emit_scan(&S, &R, &p, m->Fstar, m->Lstar);
      p.E = Epkt;
      randomdirection(&R, &p.vx, &p.vy, &p.vz);
      if ((p.x * p.vx + p.y * p.vy) + p.z * p.vz < 0.0) {
        p.vx = -p.vx;
        p.vy = -p.vy;
        p.vz = -p.vz;
      }
      p.edgeNr = 1;
      p.onEdge = 1;
      double ct = fabs(p.z) / m->R[0];
      p.i = 0;
      p.j = -1;
      for (int j = 1; j <= nt - 1; ++j)
        if (ct < m->Theta[j - 1] && ct > m->Theta[j]) p.j = j;
      if (p.j < 0) {
        for (int j = 1; j <= nt - 1; ++j)
          if (ct >= m->Theta[j]) {
            p.j = j;
            break;
          }
        if (p.j < 0) p.j = nt - 1;
      }
      if (S.scattering) {
        p.pol = 0;
        p.scatt = 0;
        p.Q = p.U = p.V = 0.0;
        set_s_from_v(&p);
      }
      double tau = -dm_log(rnd(&R));
      for (;;) {
        int st = trace2d(&S, &R, &p, tau, ip);
        if (st < 0) {
          status = 1;
          out->counters[11]++;
          done = 1;
          break;
        }
        if (st == 2) {
          out->counters[5]++;
          break; /* re-launch this packet from the star */
        }
        if (st == 1) {
          /* escape: SED bin, MCRadiation.f:576-646 (non-multiwav branch) */
          out->counters[9]++;
          double av = p.vz > 0.0 ? p.vz : -p.vz;
          int ia = (int)(av * (double)ORC_NANGLE_SED + 1.0);
          if (ia > ORC_NANGLE_SED) ia = ORC_NANGLE_SED;
          int il = (p.wl1 > p.wl2) ? p.ilam1 : p.ilam2;
          size_t k = (size_t)il * (ORC_NANGLE_SED + 1) + ia;
          double add = ((wangle[ia] * p.E) * wlam[il]) / 1.0;
          out->spec[k] += add;
          out->ispec[k] += 1;
          if (p.scatt) out->scatspec[k] += add;
          done = 1;
          break;
        }
        ninteract++;
        interact(&S, &R, &p);
        if (run->maxinteract > 0) {
          if (rnd(&R) < 1.0 / (double)run->maxinteract) {
            out->counters[7]++;
            done = 1;
            break;
          }
          p.E = (p.E * (double)run->maxinteract) / (double)(run->maxinteract - 1);
        }
        tau = -dm_log(rnd(&R));
      }
    }
  }
  for (int c = 0; c < ncell; ++c) out->T[c] = S.Tcell[c];
  free(wlam);
  free(dens);
  free(S.mass);
  free(S.Tcell);
  free(S.lastphot);
  free(S.iTD);
  free(S.kdext);
  free(S.kdabs);
  return status;
}

/* InitRandomWalk thick flags (RandomWalk.f:172-190): a cell i >= 1 is thick
 * when its radial width exceeds factRW mean free paths 1/(AU KDext dens) at
 * any of iT = 100, 600, 1100, 1600. */
void orc_init_random_walk(const orc_model *m, int scat_how, double factRW, uint8_t *thick) {
  const int nc = m->nt - 1, ncell = m->nr * nc;
  int scattering = 0;
  if (scat_how != 0)
    for (size_t k = 0; k < (size_t)ncell * m->nlam; ++k)
      if (m->KscaTot[k] != 0.0) {
        scattering = 1;
        break;
      }
  for (int c = 0; c < ncell; ++c) {
    int i = c / nc;
    thick[c] = 0;
    if (i < 1) continue;
    for (int iT = 100; iT <= 1600; iT += 500) {
      double kdext, kdabs;
      orc_diffcoeff_one(m, c, iT, scattering, &kdext, &kdabs);
      double lr = 1.0 / ((AU_CM * kdext) * m->dens[c]);
      if ((m->R[i + 1] - m->R[i]) > factRW * lr) thick[c] = 1;
    }
  }
}

/* ---------------------------------------------------------------- ray-traced spectrum
 * TracePath + TraceFlux (TraceMono.f:2032-2297, 8-497) for the thermal
 * emission and the star, without a scattering field, as the reference
 * orders it: the paths of all image rays are traced and stored first
 * (count2dpath, trace2dpath), then integrated per wavelength.  The tau =
 * 0.1 radius uses the opacities at lam_path (the reference's trace reads
 * the last packet's opacities).  exp, cos and sin of the ray set-up and the
 * attenuation are detmath's. */

typedef struct {
  int n, cap, hitstar;
  int *i, *j, *irg, *jphi1, *jphi2, *k; /* the last four with a scattered-light field */
  double *v;
} orc_path;

static void path_push(orc_path *p, int i, int j, double v) {
  if (p->n == p->cap) {
    p->cap = p->cap ? 2 * p->cap : 64;
    p->i = (int *)realloc(p->i, sizeof(int) * p->cap);
    p->j = (int *)realloc(p->j, sizeof(int) * p->cap);
    p->irg = (int *)realloc(p->irg, sizeof(int) * p->cap);
    p->jphi1 = (int *)realloc(p->jphi1, sizeof(int) * p->cap);
    p->jphi2 = (int *)realloc(p->jphi2, sizeof(int) * p->cap);
    p->k = (int *)realloc(p->k, sizeof(int) * p->cap);
    p->v = (double *)realloc(p->v, sizeof(double) * p->cap);
  }
  p->i[p->n] = i;
  p->j[p->n] = j;
  p->irg[p->n] = 1;
  p->jphi1[p->n] = p->jphi2[p->n] = 1;
  p->k[p->n] = 0;
  p->v[p->n] = v;
  p->n++;
}

/* the folded azimuth bin of a path point, trace2dpath TraceMono.f:2378-2382 */
static int path_jphi(double x, double y) {
  const double rho = sqrt(x * x + y * y); /* a point on the axis takes phi = 0 */
  double c = rho > 0.0 ? x / rho : 1.0;
  if (c > 1.0) c = 1.0;
  if (c < -1.0) c = -1.0;
  double phi = rho > 0.0 ? (180.0 * acos(c)) / PI_D : 0.0;
  if (y < 0.0) phi = -phi;
  int j = (int)(((double)(float)180 * phi) / 360.0);
  j = j + 1;
  if (j < 1) j = 1 - j;
  if (j > 90) j = 181 - j;
  return j;
}

/* the scattered-light part of the ray tracer, defined below */
typedef struct {
  int *nrg, *off, nsub;
  double *thetrg, *thet;
} sub_t;
static void sub_build(const orc_model *m, int angular, sub_t *g);
static void sub_free(sub_t *g);
static int sub_irg(const sub_t *g, int j, double theta);
static int trace2edge_rg(mc_t *s, const sub_t *g, orc_phot *p, int irg, double *v, int *inext, int *jnext,
                         int *irgnext);

static void rt_cells(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, double lam0,
                     double *kext, double *emis) {
  const int nlam = m->nlam, ncell = m->nr * (m->nt - 1), TT = ORC_TMAX + 1;
  int l1 = 0, l2 = 1;
  double w1 = 1.0, w2 = 0.0;
  for (int i = 0; i < nlam - 1; ++i)
    if (lam0 >= m->lam[i] && lam0 <= m->lam[i + 1]) {
      l1 = i;
      l2 = i + 1;
      w1 = (m->lam[i + 1] - lam0) / (m->lam[i + 1] - m->lam[i]);
      w2 = (lam0 - m->lam[i]) / (m->lam[i + 1] - m->lam[i]);
    }
  if (lam0 >= m->lam[nlam - 1]) {
    l1 = nlam - 2;
    l2 = nlam - 1;
    w1 = 0.0;
    w2 = 1.0;
  }
  for (int c = 0; c < ncell; ++c) {
    const double *w = m->comp_w + (size_t)c * m->ncomp;
    double Kabs = 0.0, Kext = 0.0, Ksca = 0.0;
    for (int q = 0; q < m->ncomp; ++q) {
      const double *Ka = Kabs_c + (size_t)q * nlam, *Ks = Ksca_c + (size_t)q * nlam;
      Kabs = Kabs + (w1 * Ka[l1] + w2 * Ka[l2]) * w[q];
      Kext = Kext + (w1 * (Ka[l1] + Ks[l1]) + w2 * (Ka[l2] + Ks[l2])) * w[q];
      Ksca = Ksca + (w1 * Ks[l1] + w2 * Ks[l2]) * w[q];
    }
    const double albedo = Ksca / Kext;
    int iT = (int)(T[c] / 1.0);
    const double wT1 = (double)(iT + 1) - T[c] / 1.0, wT2 = T[c] / 1.0 - (double)iT;
    if (iT < 1) iT = 1;
    if (iT > ORC_TMAX - 1) iT = ORC_TMAX - 1;
    double e = 0.0;
    for (int q = 0; q < m->ncomp; ++q) {
      const double *Ka = Kabs_c + (size_t)q * nlam;
      e = e + (((w1 * (wT1 * m->BB[(size_t)l1 * TT + iT] + wT2 * m->BB[(size_t)l1 * TT + iT + 1])) * Ka[l1] +
                (w2 * (wT1 * m->BB[(size_t)l2 * TT + iT] + wT2 * m->BB[(size_t)l2 * TT + iT + 1])) * Ka[l2]) *
               w[q]) / Kabs;
    }
    kext[c] = Kext;
    emis[c] = e * (1.0 - albedo);
  }
}

static void sel_sort(double *x, int n) { /* sort, Subroutines.f:1907-1927 */
  for (int j = 0; j < n - 1; ++j) {
    double mn = x[j];
    int im = j;
    for (int i = j; i < n; ++i)
      if (x[i] < mn) {
        mn = x[i];
        im = i;
      }
    mn = x[j];
    x[j] = x[im];
    x[im] = mn;
  }
}

static int trace_run(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, int scat_how,
                     double angle, int nphi, int nj0, int nRfix, const double *Rfix, double lam_path, int tracestar,
                     double dimstar, int nobs, const double *lam_obs, double *flux, int *info, double **Ri_out,
                     double **image_out, const orc_scat_opts *so);

int orc_trace_spectrum(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T,
                       int scat_how, double angle, int nphi, int nj0, int nRfix, const double *Rfix,
                       double lam_path, int tracestar, double dimstar, int nobs, const double *lam_obs, double *flux,
                       int *info) {
  return trace_run(m, Kabs_c, Ksca_c, T, scat_how, angle, nphi, nj0, nRfix, Rfix, lam_path, tracestar, dimstar, nobs,
                   lam_obs, flux, info, NULL, NULL, NULL);
}

int orc_trace_spectrum_scat(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T,
                            int scat_how, double angle, int nphi, int nj0, int nRfix, const double *Rfix,
                            double lam_path, int tracestar, double dimstar, int nobs, const double *lam_obs,
                            double *flux, int *info, const orc_scat_opts *so) {
  return trace_run(m, Kabs_c, Ksca_c, T, scat_how, angle, nphi, nj0, nRfix, Rfix, lam_path, tracestar, dimstar, nobs,
                   lam_obs, flux, info, NULL, NULL, so);
}

/* TracePath + TraceFlux (TraceMono.f:2032-2297, 8-497); when Ri_out and
 * image_out are given they receive (malloc'ed) the image radii and the last
 * wavelength's intensities, radius-major.  so (may be NULL): the
 * scattered-light field's settings; with packets and a scattering model
 * each wavelength gets its field (orc_scatter_field, keys seed, seed+1, ...
 * in the order the fields are made; isotropic models one per grid
 * wavelength, made when first needed) and the formal solution adds twice
 * its source (TraceMono.f:356-395); a full-Mueller model's paths then step
 * through the sub-cones with Trace2edgeRG. */
static int trace_run(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, int scat_how,
                     double angle, int nphi, int nj0, int nRfix, const double *Rfix, double lam_path, int tracestar,
                     double dimstar, int nobs, const double *lam_obs, double *flux, int *info, double **Ri_out,
                     double **image_out, const orc_scat_opts *so) {
  const int nR = m->nr, nTheta = m->nt, nc = nTheta - 1, ncell = nR * nc, nstar = 30;
  mc_t s;
  memset(&s, 0, sizeof s);
  s.m = m;
  s.nc = nc;
  int smode = 0;
  if (so && (so->nphot > 0 || so->nstar > 0) && (scat_how == 1 || scat_how == 2)) {
    for (int q = 0; q < m->ncomp * m->nlam; ++q)
      if (Ksca_c[q] > 0.0) smode = scat_how;
  }
  sub_t g;
  memset(&g, 0, sizeof g);
  if (smode) sub_build(m, smode == 2, &g);
  double *kext = (double *)malloc(sizeof(double) * ncell), *emis = (double *)malloc(sizeof(double) * ncell);
  /* tau01R, midplane direction */
  rt_cells(m, Kabs_c, Ksca_c, T, lam_path, kext, emis);
  double R01;
  {
    const double r = m->R[1], ct = (m->Theta[nc - 1] + m->Theta[nc]) / 2.0;
    orc_phot p;
    memset(&p, 0, sizeof p);
    p.x = sqrt(1.0 - ct * ct) * r;
    p.z = ct * r;
    p.edgeNr = 1;
    p.onEdge = 1;
    p.vx = p.x / r;
    p.vz = p.z / r;
    p.i = 1;
    p.j = nc;
    double tau = 0.0, v;
    int escape = 0, inext, jnext;
    for (int n = 0; n < 1000000; ++n) {
      if (trace2edge(&s, &p, &v, &inext, &jnext) != 0) break;
      const int c = p.i * nc + (p.j - 1);
      const double tau1 = ((kext[c] * v) * m->dens[c]) * AU_CM;
      if (tau + tau1 > 0.1) {
        v = v * (0.1 - tau) / tau1;
        p.x = p.x + p.vx * v;
        p.y = p.y + p.vy * v;
        p.z = p.z + p.vz * v;
        break;
      }
      p.x = p.x + p.vx * v;
      p.y = p.y + p.vy * v;
      p.z = p.z + p.vz * v;
      p.onEdge = 1;
      tau = tau + tau1;
      if (inext >= nR || inext < 0) {
        escape = 1;
        break;
      }
      p.i = inext;
      p.j = jnext;
    }
    if (escape) p.z = 0.0;
    R01 = sqrt(p.x * p.x + p.z * p.z);
    if (R01 > m->R[nR - 1]) R01 = m->R[1];
  }
  /* image radii (TraceMono.f:2108-2222) */
  int nimg = (nj0 > 0 ? nj0 * (nR - 1) : (nR - 2) / (-nj0) + 1) + nc * 2 * (nRfix + 2) + 1 + nstar;
  if (scat_how == 2) nimg += 180 * (nRfix + 1);
  double *Ri = (double *)calloc((size_t)nimg, sizeof(double));
  double *ta = (double *)malloc(sizeof(double) * (nTheta + 1));
  for (int j = 1; j <= nc; ++j) ta[j] = acos((m->Theta[j - 1] + m->Theta[j]) / 2.0);
  int nj = 0;
  for (int j = 1; j <= nc; ++j) {
    Ri[nj++] = R01 * fabs(cos(PI_D / 2.0 - ta[j] + angle));
    Ri[nj++] = fabs(R01 * cos(ta[j] - PI_D / 2.0 + angle));
  }
  for (int j = 1; j <= nc; ++j) {
    Ri[nj++] = R01 * fabs(cos(PI_D / 2.0 - ta[j]));
    Ri[nj++] = fabs(R01 * cos(ta[j] - PI_D / 2.0));
  }
  if (scat_how == 2)
    for (int j = 1; j <= 180; ++j) {
      const double theta = (double)(float)j * (PI_D / 2.0) / 181.0;
      Ri[nj++] = m->R[1] * fabs(cos(PI_D / 2.0 - theta));
      for (int i = 0; i < nRfix; ++i) Ri[nj++] = Rfix[i] * fabs(cos(PI_D / 2.0 - theta));
    }
  for (int i = 0; i < nRfix; ++i)
    for (int j = 1; j <= nc; ++j) {
      Ri[nj++] = Rfix[i] * fabs(cos(PI_D / 2.0 - ta[j] + angle));
      Ri[nj++] = fabs(Rfix[i] * cos(ta[j] - PI_D / 2.0 + angle));
    }
  sel_sort(Ri, nj);
  if (nj0 > 0) {
    for (int i = 1; i <= nR - 1; ++i)
      for (int j = 1; j <= nj0; ++j)
        Ri[nj++] = m->R[i] + (m->R[i + 1] - m->R[i]) * ((double)(float)j - 0.5) / (double)(float)nj0;
  } else {
    for (int i = 1; i <= nR - 1; i += -nj0) Ri[nj++] = pow(10.0, log10(m->R[i] * m->R[i + 1]) / 2.0);
  }
  for (int i = 1; i <= nstar - 1; ++i) Ri[nj++] = ((0.999 * m->R[0]) * (double)(float)(i - 1)) / (double)(float)(nstar - 2);
  Ri[nj++] = m->R[0] * (double)1.001f;
  Ri[nimg - 1] = m->R[nR] * (double)0.9999f;
  sel_sort(Ri, nimg);
  {
    int k = 0;
  restart:
    k = k + 1;
    for (int i = nimg - 1; i >= 1; --i)
      if (Ri[i] == Ri[i - 1]) {
        if (i != nimg - 1)
          Ri[i] = (Ri[i + 1] + Ri[i]) / 2.0;
        else
          Ri[i - 1] = (Ri[i - 1] + Ri[i]) / 2.0;
        if (k < nimg * 10) goto restart;
      }
  }
  /* paths (TraceMono.f:2236-2290, trace2dpath) */
  orc_path *paths = (orc_path *)calloc((size_t)nimg * nphi, sizeof(orc_path));
  double *phi = (double *)malloc(sizeof(double) * nphi);
  int bad = 0;
  for (int i = 0; i < nimg; ++i)
    for (int k = 1; k <= nphi; ++k) {
      phi[k - 1] = 1e-5 + PI_D * (double)((float)k - 0.5f) / (double)(float)nphi;
      const double Rad = Ri[i], Rout = m->R[nR];
      orc_phot p;
      memset(&p, 0, sizeof p);
      p.x = Rad * dm_cos(phi[k - 1]);
      p.y = Rad * dm_sin(phi[k - 1]);
      p.z = sqrt(Rout * Rout - Rad * Rad);
      p.edgeNr = 2;
      p.onEdge = 1;
      rotate(&p.x, &p.y, &p.z, 0.0, 1.0, 0.0, angle);
      const double ct = fabs(p.z) / Rout;
      p.i = nR - 1;
      p.j = 1;
      for (int j = 1; j <= nc; ++j)
        if (ct < m->Theta[j - 1] && ct >= m->Theta[j]) p.j = j;
      int irg = smode == 2 ? sub_irg(&g, p.j, acos(ct)) : 1;
      p.vx = 0.0;
      p.vy = 0.0;
      p.vz = -1.0;
      rotate(&p.vx, &p.vy, &p.vz, 0.0, 1.0, 0.0, angle);
      orc_path *pa = &paths[(size_t)i * nphi + (k - 1)];
      for (int n = 0;; ++n) {
        double v;
        int inext, jnext, irgn = irg;
        const int f = smode == 2 ? trace2edge_rg(&s, &g, &p, irg, &v, &inext, &jnext, &irgn)
                                 : trace2edge(&s, &p, &v, &inext, &jnext);
        if (n >= (1 << 20) || f != 0) {
          bad++;
          break;
        }
        p.onEdge = 1;
        path_push(pa, p.i, p.j, v);
        const int q = pa->n - 1;
        pa->irg[q] = irg;
        if (smode) pa->jphi1[q] = path_jphi(p.x, p.y);
        p.x = p.x + p.vx * v;
        p.y = p.y + p.vy * v;
        p.z = p.z + p.vz * v;
        if (smode) {
          pa->jphi2[q] = path_jphi(p.x, p.y);
          pa->k[q] = p.z > 0.0 ? 0 : 1;
        }
        if (inext >= nR) break;
        if (inext < 0) {
          pa->hitstar = 1;
          break;
        }
        p.i = inext;
        p.j = jnext;
        irg = irgn;
      }
    }
  /* TraceFlux per wavelength */
  double *image = (double *)calloc((size_t)nimg * nphi, sizeof(double));
  size_t flen = smode ? (size_t)nR * g.nsub * 2 * 91 : 0;
  double *SF = smode ? (double *)malloc(sizeof(double) * flen) : NULL, *alb = (double *)malloc(sizeof(double) * ncell);
  double **iso = smode == 1 ? (double **)calloc((size_t)m->nlam, sizeof(double *)) : NULL;
  double *fracirg = NULL;
  uint64_t nfields = 0;
  if (smode) {
    fracirg = (double *)malloc(sizeof(double) * g.nsub);
    for (int j = 1; j <= nc; ++j) {
      const int kq = g.nrg[j - 1];
      const double dth = (g.thet[j] - g.thet[j - 1]) / (double)(float)kq;
      for (int q = 1; q <= kq; ++q)
        fracirg[g.off[j - 1] + q - 1] = (cos(g.thet[j - 1] + (double)(float)(q - 1) * dth) -
                                         cos(g.thet[j - 1] + (double)(float)q * dth)) /
                                        (m->Theta[j - 1] - m->Theta[j]);
    }
  }
  int64_t finfo[4];
  for (int l = 0; l < nobs; ++l) {
    const double lam0 = lam_obs[l];
    flux[l] = 0.0;
    if (lam0 < m->lam[0] || lam0 > m->lam[m->nlam - 1]) continue;
    int l1 = 0, l2 = 1;
    double w1 = 1.0, w2 = 0.0;
    for (int i = 0; i < m->nlam - 1; ++i)
      if (lam0 >= m->lam[i] && lam0 <= m->lam[i + 1]) {
        l1 = i;
        l2 = i + 1;
        w1 = (m->lam[i + 1] - lam0) / (m->lam[i + 1] - m->lam[i]);
        w2 = (lam0 - m->lam[i]) / (m->lam[i + 1] - m->lam[i]);
      }
    if (lam0 >= m->lam[m->nlam - 1]) {
      l1 = m->nlam - 2;
      l2 = m->nlam - 1;
      w1 = 0.0;
      w2 = 1.0;
    }
    rt_cells(m, Kabs_c, Ksca_c, T, lam0, kext, emis);
    const double *F1 = NULL, *F2 = NULL;
    if (smode) {
      for (int c = 0; c < ncell; ++c) { /* TraceFlux's albedo at lam0 */
        const double *w = m->comp_w + (size_t)c * m->ncomp;
        double Ke = 0.0, Ks = 0.0;
        for (int q = 0; q < m->ncomp; ++q) {
          const double *a = Kabs_c + (size_t)q * m->nlam, *sk = Ksca_c + (size_t)q * m->nlam;
          Ke = Ke + (w1 * (a[l1] + sk[l1]) + w2 * (a[l2] + sk[l2])) * w[q];
          Ks = Ks + (w1 * sk[l1] + w2 * sk[l2]) * w[q];
        }
        alb[c] = Ks / Ke;
      }
      if (smode == 2) {
        orc_scatter_field(m, Kabs_c, Ksca_c, T, scat_how, angle, lam0, so->nphot, so->nstar, so->seed + nfields++,
                          so->nexits, SF, finfo);
        F1 = F2 = SF;
      } else {
        const int ls[2] = {l1, l2};
        for (int q = 0; q < 2; ++q)
          if (!iso[ls[q]]) {
            iso[ls[q]] = (double *)malloc(sizeof(double) * flen);
            orc_scatter_field(m, Kabs_c, Ksca_c, T, scat_how, angle, m->lam[ls[q]], so->nphot, so->nstar,
                              so->seed + nfields++, so->nexits, iso[ls[q]], finfo);
          }
        F1 = iso[l1];
        F2 = iso[l2];
      }
    }
    for (int i = 0; i < nimg; ++i)
      for (int k = 0; k < nphi; ++k) {
        const orc_path *pa = &paths[(size_t)i * nphi + k];
        double I = 0.0, tau = 0.0, fact = 1.0;
        int stopped = 0;
        for (int q = 0; q < pa->n; ++q) {
          const int ip = pa->i[q], jp = pa->j[q];
          if (ip != 0) {
            const int c = ip * nc + (jp - 1);
            const double tau_e = ((pa->v[q] * m->dens[c]) * kext[c]) * AU_CM;
            double src = emis[c];
            if (smode) {
              double xs = 0.0;
              const int kp = pa->k[q];
              if (smode == 2) {
                const int irg = pa->irg[q], sub = g.off[jp - 1] + (irg - 1);
                const size_t base = (((size_t)ip * g.nsub + sub) * 2 + kp) * 91;
                const double ww = alb[c] / (m->V[c] * fracirg[sub]);
                const int jj1 = pa->jphi1[q], jj2 = pa->jphi2[q], djj = jj1 <= jj2 ? 1 : -1;
                int njj = 0;
                for (int jj = jj1;; jj += djj) {
                  xs = xs + ww * F1[base + jj];
                  ++njj;
                  if (jj == jj2) break;
                }
                xs = xs / (double)(float)njj;
              } else {
                const size_t b = ((size_t)c * 2 + kp) * 91;
                xs = ((w1 * F1[b] + w2 * F2[b]) / m->V[c]) * alb[c];
              }
              src = 2.0 * xs + emis[c];
            }
            if (tau_e < 1e-6) {
              I = I + (src * tau_e) * fact;
              fact = fact * (1.0 - tau_e);
            } else {
              const double ex = dm_exp(-tau_e);
              I = I + (src * (1.0 - ex)) * fact;
              fact = fact * ex;
            }
            tau = tau + tau_e;
          }
          if (tau > 1e8) {
            stopped = 1;
            break;
          }
        }
        if (!stopped && pa->hitstar && tracestar)
          I = I + (((m->Fstar[l1] * w1 + m->Fstar[l2] * w2) * fact) * dimstar) /
                      (PI_D * ((m->R[0] * AU_CM) * (m->R[0] * AU_CM)));
        image[(size_t)i * nphi + k] = I;
      }
    double f = 0.0;
    for (int i = 0; i < nimg - 1; ++i)
      for (int k = 0; k < nphi; ++k) {
        const double w1a = (((2.0 * PI_D) * fabs(Ri[i])) * (AU_CM * AU_CM)) / (double)(float)nphi;
        const double w2a = (((2.0 * PI_D) * fabs(Ri[i + 1])) * (AU_CM * AU_CM)) / (double)(float)nphi;
        f = f + ((Ri[i + 1] - Ri[i]) * (w1a * image[(size_t)i * nphi + k] + w2a * image[(size_t)(i + 1) * nphi + k])) / 2.0;
      }
    flux[l] = f;
  }
  info[0] = nimg;
  info[1] = bad;
  for (int q = 0; q < nimg * nphi; ++q) {
    free(paths[q].i);
    free(paths[q].j);
    free(paths[q].irg);
    free(paths[q].jphi1);
    free(paths[q].jphi2);
    free(paths[q].k);
    free(paths[q].v);
  }
  free(SF);
  free(alb);
  free(fracirg);
  if (iso) {
    for (int l = 0; l < m->nlam; ++l) free(iso[l]);
    free(iso);
  }
  if (smode) sub_free(&g);
  free(paths); free(phi); free(ta); free(kext); free(emis);
  if (Ri_out && image_out) {
    *Ri_out = Ri;
    *image_out = image;
  } else {
    free(Ri);
    free(image);
  }
  return 0;
}

/* MakeImage (TraceMono.f:2759-3001) for an image without polarisation,
 * planets or convolution.  Loop order i (image ring), j (angle column), k
 * (point), as the reference's single-threaded run; point s = (i nphi + j)
 * nint + k takes its two uniforms from one Philox block with key seed and
 * counter (0, 1, s_lo, s_hi).  The interpolation is the 10**() of the
 * interpolated log10 I (TraceMono.f:2931-2934), evaluated as exp of the
 * interpolated natural logarithm, or linear (linear != 0: the value the
 * polarised branch falls back to when Q = U = V = 0, TraceMono.f:2901-2920).
 * im[(ix-1) npix + (iy-1)]. */
int orc_trace_image(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, int scat_how,
                    double angle, int nphi, int nj0, int nRfix, const double *Rfix, int tracestar, double dimstar,
                    double lam0, int npix, int nint, double Rmax, double pa, uint64_t seed, int linear, double *flux,
                    double *im, int *info) {
  return orc_trace_image_scat(m, Kabs_c, Ksca_c, T, scat_how, angle, nphi, nj0, nRfix, Rfix, tracestar, dimstar, lam0,
                              npix, nint, Rmax, pa, seed, linear, flux, im, info, NULL);
}

int orc_trace_image_scat(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T,
                         int scat_how, double angle, int nphi, int nj0, int nRfix, const double *Rfix, int tracestar,
                         double dimstar, double lam0, int npix, int nint, double Rmax, double pa, uint64_t seed,
                         int linear, double *flux, double *im, int *info, const orc_scat_opts *so) {
  double *Ri = NULL, *image = NULL;
  trace_run(m, Kabs_c, Ksca_c, T, scat_how, angle, nphi, nj0, nRfix, Rfix, lam0, tracestar, dimstar, 1, &lam0, flux,
            info, &Ri, &image, so);
  const int nimg = info[0];
  memset(im, 0, sizeof(double) * (size_t)npix * npix);
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  long long s = 0;
  for (int i = 1; i <= nimg - 1; ++i)
    for (int j = 1; j <= nphi; ++j) {
      const double w2 = (((2.0 * PI_D) * (AU_CM * AU_CM)) * (Ri[i] - Ri[i - 1])) / (double)(float)nphi;
      for (int k = 1; k <= nint; ++k, ++s) {
        const uint32_t ctr[4] = {0u, 1u, (uint32_t)s, (uint32_t)((unsigned long long)s >> 32)};
        uint32_t o[4];
        px_philox4x32_10(ctr, key, o);
        const double ranR = px_u01(o[0], o[1]), ranPhi = px_u01(o[2], o[3]);
        const double R = Ri[i - 1] + (Ri[i] - Ri[i - 1]) * ranR;
        const double phi = (PI_D * ((double)(float)(j - 1) + ranPhi)) / (double)(float)nphi;
        int jp1, jp2;
        double wp1, wp2;
        if (ranPhi < 0.5) {
          wp1 = 0.5 - ranPhi;
          jp1 = j - 1;
          if (jp1 == 0) jp1 = 1;
          wp2 = ranPhi + 0.5;
          jp2 = j;
        } else {
          wp1 = ranPhi - 0.5;
          jp1 = j + 1;
          if (jp1 == nphi + 1) jp1 = nphi;
          wp2 = 1.5 - ranPhi;
          jp2 = j;
        }
        const double wr1 = 1.0 - ranR, wr2 = ranR;
        /* image(ir, jp) of the reference, ir = i, i+1 (1-based) */
        const double I11 = image[(size_t)(i - 1) * nphi + (jp1 - 1)], I12 = image[(size_t)(i - 1) * nphi + (jp2 - 1)];
        const double I21 = image[(size_t)i * nphi + (jp1 - 1)], I22 = image[(size_t)i * nphi + (jp2 - 1)];
        double f;
        if (linear) {
          f = ((wr1 * (wp1 * I11 + wp2 * I12) + wr2 * (wp1 * I21 + wp2 * I22)) * w2) * R;
        } else {
          f = wr1 * (wp1 * dm_log(I11) + wp2 * dm_log(I12)) + wr2 * (wp1 * dm_log(I21) + wp2 * dm_log(I22));
          f = (dm_exp(f) * w2) * R;
        }
        const double add = f / (double)(float)(2 * nint);
        for (int side = 0; side < 2; ++side) {
          const double a = side == 0 ? phi + (pa * PI_D) / 180.0 : -phi + (pa * PI_D) / 180.0;
          double x = -R * dm_cos(a);
          x = (((double)(float)npix * (x + Rmax)) / (2.0 * Rmax)) + 1.0;
          double y = R * dm_sin(a);
          y = (((double)(float)npix * (y + Rmax)) / (2.0 * Rmax)) + 1.0;
          /* ix = x truncates toward zero; kept when 1 <= ix <= npix */
          if (x >= 1.0 && x < (double)npix + 1.0 && y >= 1.0 && y < (double)npix + 1.0) {
            const int ix = (int)x, iy = (int)y;
            im[(size_t)(ix - 1) * npix + (iy - 1)] = im[(size_t)(ix - 1) * npix + (iy - 1)] + add;
          }
        }
      }
    }
  free(Ri);
  free(image);
  return 0;
}

/* ------------------------------------------------------------------------
 * The scattered-light field of the ray tracer: TraceMono (TraceMono.f:583-
 * 914) for one wavelength and inclination, single-threaded, packet after
 * packet as the reference's loop runs: the cells' opacities and mixed
 * Mueller matrices at lam0 (TraceMono.f:664-750), EmissionDistribution
 * (:956-1121; thermal contact, exit depths over nexits directions with
 * trace2exit :2659-2697), MakeStarScatter (:1585-1770), then the packets of
 * emitposition (:1124-1290) through trace2dmono (:1291-1411) with
 * makescattfield (:1416-1497) and the albedo roulette and scattering
 * (:852-880).  Theta rows are split into sub-cones for a full-Mueller
 * field (Telescope.f:93-110; thet taken as acos(Theta)) and traced with
 * Trace2edgeRG (:2487-2657).
 *
 * Random numbers: starlight packet w draws the Philox stream (key, w),
 * Monte Carlo packet w the stream (key, nstar + w), where the reference
 * continues ran2.  Albedo**0.25 is taken as two square roots, exp, log, sin
 * and cos are detmath's, acos is the C library's.  SF: nR*nsub*2*91, laid
 * out as mcg_scatter_field documents.  info: [0] nsub, [1] geometry
 * failures, [2] interaction-cap kills, [3] packets with no start. */

#define SF_NPHI_O 180
#define SF_NB_O 91

static void sub_build(const orc_model *m, int angular, sub_t *g) {
  const int nt = m->nt, nc = nt - 1;
  g->thet = (double *)malloc(sizeof(double) * nt);
  for (int j = 0; j < nt; ++j) g->thet[j] = acos(m->Theta[j]);
  g->thet[0] = 0.0;
  g->thet[nt - 1] = PI_D / 2.0;
  g->nrg = (int *)malloc(sizeof(int) * nc);
  g->off = (int *)malloc(sizeof(int) * nc);
  int n = 0;
  for (int j = 1; j <= nc; ++j) {
    int k = 1;
    if (angular) {
      const int q = (int)((g->thet[j] - g->thet[j - 1]) * 270.0 / PI_D);
      if (q > 1) k = q;
    }
    g->nrg[j - 1] = k;
    g->off[j - 1] = n;
    n += k;
  }
  g->nsub = n;
  g->thetrg = (double *)malloc(sizeof(double) * (size_t)(n + nc));
  for (int j = 1; j <= nc; ++j) {
    const int k = g->nrg[j - 1];
    double *tr = g->thetrg + g->off[j - 1] + (j - 1);
    for (int q = 1; q <= k + 1; ++q) {
      const double c = cos(g->thet[j - 1] + (double)(float)(q - 1) * ((g->thet[j] - g->thet[j - 1]) / (double)(float)k));
      tr[q - 1] = c * c;
    }
    tr[0] = m->Theta[j - 1] * m->Theta[j - 1];
    tr[k] = m->Theta[j] * m->Theta[j];
  }
}

static void sub_free(sub_t *g) {
  free(g->nrg); free(g->off); free(g->thetrg); free(g->thet);
}

static int sub_irg(const sub_t *g, int j, double theta) {
  const int k = g->nrg[j - 1];
  if (k <= 1 || !(theta == theta)) return 1;
  int irg = (int)((double)(float)k * (theta - g->thet[j - 1]) / (g->thet[j] - g->thet[j - 1])) + 1;
  if (irg > k) irg = k;
  if (irg < 1) irg = 1;
  return irg;
}

/* Trace2edgeRG, TraceMono.f:2487-2657 */
static int trace2edge_rg(mc_t *s, const sub_t *g, orc_phot *p, int irg, double *v, int *inext, int *jnext,
                         int *irgnext) {
  const orc_model *m = s->m;
  const int nt = m->nt, nrg = g->nrg[p->j - 1];
  double r = (p->x * p->x + p->y * p->y) + p->z * p->z;
  double R1 = m->R[p->i] * m->R[p->i], R2 = m->R[p->i + 1] * m->R[p->i + 1], T1, T2;
  if (nrg <= 1) {
    T1 = m->Theta[p->j - 1] * m->Theta[p->j - 1];
    T2 = m->Theta[p->j] * m->Theta[p->j];
  } else {
    T1 = g->thetrg[g->off[p->j - 1] + (p->j - 1) + irg - 1];
    T2 = g->thetrg[g->off[p->j - 1] + (p->j - 1) + irg];
  }
  double b = 2.0 * ((p->x * p->vx + p->y * p->vy) + p->z * p->vz);
  int hitR1, hitR2, hitT1, hitT2;
  double vR1, vR2, vT1, vT2;
  if (!p->onEdge) {
    hitR1 = hitR(R1, r, b, &vR1);
    hitR2 = hitR(R2, r, b, &vR2);
    hitT1 = hitT(p, T1, r, b, &vT1);
    hitT2 = hitT(p, T2, r, b, &vT2);
  } else if (p->edgeNr == 1) {
    hitR1 = 0;
    vR1 = 1e200;
    hitR2 = hitR(R2, r, b, &vR2);
    hitT1 = hitT(p, T1, r, b, &vT1);
    hitT2 = hitT(p, T2, r, b, &vT2);
  } else if (p->edgeNr == 2) {
    hitR1 = hitR(R1, r, b, &vR1);
    hitR2 = 1;
    vR2 = -b;
    hitT1 = hitT(p, T1, r, b, &vT1);
    hitT2 = hitT(p, T2, r, b, &vT2);
  } else if (p->edgeNr == 3) {
    hitR1 = hitR(R1, r, b, &vR1);
    hitR2 = hitR(R2, r, b, &vR2);
    hitT1 = 0;
    vT1 = 1e200;
    if (p->j != nt - 1 || irg != nrg) {
      hitT2 = hitT(p, T2, r, b, &vT2);
    } else {
      vT2 = -p->z / p->vz;
      hitT2 = vT2 > 0.0;
    }
  } else {
    hitR1 = hitR(R1, r, b, &vR1);
    hitR2 = hitR(R2, r, b, &vR2);
    if (p->j != 1 || irg != 1) {
      hitT1 = hitT(p, T1, r, b, &vT1);
    } else {
      hitT1 = 0;
      vT1 = 1e200;
    }
    if (p->j != nt - 1 || irg != nrg) {
      hitT2 = hitTsame(p, T2, b, &vT2);
    } else {
      hitT2 = 0;
      vT2 = 1e200;
    }
  }
  if (!hitR1 && !hitR2 && !hitT1 && !hitT2) {
    hitR1 = hitR(R1, r, b, &vR1);
    hitR2 = hitR(R2, r, b, &vR2);
    hitT1 = hitT(p, T1, r, b, &vT1);
    hitT2 = hitT(p, T2, r, b, &vT2);
    if (!hitR1 && !hitR2 && !hitT1 && !hitT2) return 1;
  }
  *v = 1e200;
  *inext = p->i;
  *jnext = p->j;
  *irgnext = irg;
  if (hitR1 && vR1 < *v) {
    *v = vR1;
    *inext = p->i - 1;
    *jnext = p->j;
    *irgnext = irg;
    p->edgeNr = 2;
  }
  if (hitR2 && vR2 < *v) {
    *v = vR2;
    *inext = p->i + 1;
    *jnext = p->j;
    *irgnext = irg;
    p->edgeNr = 1;
  }
  if (hitT1 && vT1 < *v) {
    *v = vT1;
    *inext = p->i;
    if (nrg > 1) {
      *irgnext = irg - 1;
      *jnext = p->j;
      if (*irgnext < 1) {
        *jnext = p->j - 1;
        *irgnext = *jnext > 0 ? g->nrg[*jnext - 1] : 1;
      }
    } else {
      *jnext = p->j - 1;
      if (*jnext > 0) *irgnext = g->nrg[*jnext - 1];
    }
    p->edgeNr = 4;
  }
  if (hitT2 && vT2 < *v) {
    *v = vT2;
    *inext = p->i;
    if (nrg > 1) {
      *irgnext = irg + 1;
      *jnext = p->j;
      if (*irgnext > nrg) {
        *jnext = p->j + 1;
        *irgnext = 1;
        if (*jnext == nt) *irgnext = g->nrg[nt - 2];
      }
    } else {
      *jnext = p->j + 1;
      *irgnext = 1;
    }
    p->edgeNr = 3;
  }
  if (*jnext == nt) {
    *jnext = nt - 1;
    *irgnext = g->nrg[nt - 2];
    p->edgeNr = 4;
  }
  if (*jnext == 0) {
    *jnext = 1;
    *irgnext = 1;
    p->edgeNr = 3;
  }
  return 0;
}

typedef struct {
  mc_t s;
  sub_t g;
  int mode, nc;
  double *kabs, *kext, *alb, *F, *vis, *cum, *dirs, *SF;
  long ncum;
  double Etot, Estar;
  int64_t nstar, nphot;
  int64_t *info;
} sf_run;

static size_t sf_base_o(const sf_run *q, int i, int j, int irg, int side) {
  return (((size_t)i * q->g.nsub + q->g.off[j - 1] + (irg - 1)) * 2 + side) * SF_NB_O;
}

/* the 180 observer directions' angle indices and rotated Q of a flight */
static void sf_dirs_o(const sf_run *q, const orc_phot *p, int *ia, double *Qd) {
  for (int k = 0; k < SF_NPHI_O; ++k) {
    const double sx = q->dirs[3 * k], sy = q->dirs[3 * k + 1], sz = q->dirs[3 * k + 2];
    double c = (p->vx * sx + p->vy * sy) + p->vz * sz;
    if (c > 1.0) c = 1.0;
    if (c < -1.0) c = -1.0;
    int a = (int)((180.0 * acos(c)) / PI_D + 1.0);
    if (a > 180) a = 180;
    if (a < 1) a = 1;
    ia[k] = a - 1;
    Qd[k] = p->Q;
    if (p->pol) {
      double xn = p->vy * sz - p->vz * sy, yn = p->vz * sx - p->vx * sz, zn = p->vx * sy - p->vy * sx;
      const double r = sqrt((xn * xn + yn * yn) + zn * zn);
      if (r > 0.0) {
        orc_phot t = *p;
        rotate_stokes(&t, xn / r, yn / r, zn / r);
        Qd[k] = t.Q;
      }
    }
  }
}

/* the folded azimuth deposits of a segment, loop order i = 1..180 */
static void sf_fold_o(sf_run *q, size_t base, const double *Fc, double x, double y, double E, double vAU,
                      const int *ia, const double *Qd, int withQ) {
  const double rho = sqrt(x * x + y * y);
  double phi0 = rho > 0.0 ? (180.0 * acos(x / rho)) / PI_D : 0.0;
  if (y < 0.0) phi0 = 360.0 - phi0;
  const double phi = 180.0 / (double)(float)SF_NPHI_O;
  int j = (int)(((double)(float)SF_NPHI_O * (phi + phi0)) / 360.0);
  for (int i = 1; i <= SF_NPHI_O; ++i) {
    if (j < 1) j = j + SF_NPHI_O;
    if (j > SF_NPHI_O) j = j - SF_NPHI_O;
    const int a = ia[j - 1];
    const double sI = withQ ? Fc[a] * E + Fc[180 + a] * Qd[j - 1] : Fc[a] * E;
    const int bin = i <= SF_NPHI_O / 2 ? i : SF_NPHI_O + 1 - i;
    q->SF[base + bin] = q->SF[base + bin] + sI * vAU;
    j = j + 1;
  }
}

static int sf_star_start_o(sf_run *q, rng_t *r, orc_phot *p, int *irg, int byct) {
  const orc_model *m = q->s.m;
  const double R0 = m->R[0];
  randomdirection(r, &p->x, &p->y, &p->z);
  p->x = R0 * p->x;
  p->y = R0 * p->y;
  p->z = R0 * p->z;
  randomdirection(r, &p->vx, &p->vy, &p->vz);
  const double inp = (p->x * p->vx + p->y * p->vy) + p->z * p->vz;
  if (inp < 0.0) {
    p->vx = -p->vx;
    p->vy = -p->vy;
    p->vz = -p->vz;
  }
  p->edgeNr = 1;
  p->onEdge = 1;
  const double ct = fabs(p->z) / R0;
  for (int j = 1; j <= q->nc; ++j)
    if (ct < m->Theta[j - 1] && ct > m->Theta[j]) {
      p->i = 0;
      p->j = j;
      *irg = sub_irg(&q->g, j, acos(byct ? ct : fabs(p->z) / sqrt((p->x * p->x + p->y * p->y) + p->z * p->z)));
      return 1;
    }
  return 0;
}

static void sf_star_packet(sf_run *q, uint64_t key, int64_t w) {
  const orc_model *m = q->s.m;
  const int nc = q->nc;
  rng_t r;
  memset(&r, 0, sizeof r);
  px_init(&r.px, key, (uint64_t)w);
  orc_phot p;
  memset(&p, 0, sizeof p);
  int irg = 1, ia[SF_NPHI_O];
  double Qd[SF_NPHI_O];
  p.E = q->Estar / (double)(float)q->nstar;
  if (!sf_star_start_o(q, &r, &p, &irg, 1)) {
    const double ct = fabs(p.z) / m->R[0];
    p.i = 0;
    p.j = 1;
    for (int j = 1; j <= nc; ++j)
      if (ct <= m->Theta[j - 1] && ct >= m->Theta[j]) {
        p.j = j;
        break;
      }
    irg = sub_irg(&q->g, p.j, acos(ct));
  }
  if (q->mode == 2) sf_dirs_o(q, &p, ia, Qd);
  for (int n = 0;; ++n) {
    double v;
    int inext, jnext, irgn;
    if (n >= (1 << 20) || trace2edge_rg(&q->s, &q->g, &p, irg, &v, &inext, &jnext, &irgn) != 0) {
      q->info[1]++;
      return;
    }
    const size_t c = (size_t)p.i * nc + (p.j - 1);
    const double tau = (m->dens[c] * q->kext[c]) * AU_CM;
    const double w1 = (tau * v > 1e-5) ? (1.0 - dm_exp(-tau * v)) / tau : v;
    if (q->mode == 1) {
      const size_t b = sf_base_o(q, p.i, p.j, 1, 0);
      q->SF[b] = q->SF[b] + ((p.E * w1) * AU_CM) / 2.0;
      q->SF[b + SF_NB_O] = q->SF[b + SF_NB_O] + ((p.E * w1) * AU_CM) / 2.0;
    } else {
      const double x = p.x + (p.vx * v) / 2.0, y = p.y + (p.vy * v) / 2.0;
      const size_t b = sf_base_o(q, p.i, p.j, irg < 1 ? 1 : irg, p.z > 0.0 ? 0 : 1);
      q->SF[b] = q->SF[b] + (p.E * w1) * AU_CM;
      sf_fold_o(q, b, q->F + c * 1082, x, y, p.E, (v * AU_CM) / 2.0, ia, Qd, 0);
    }
    p.E = p.E * dm_exp(-tau * v);
    p.x = p.x + p.vx * v;
    p.y = p.y + p.vy * v;
    p.z = p.z + p.vz * v;
    p.onEdge = 1;
    if (inext >= m->nr || inext < 0) return;
    p.i = inext;
    p.j = jnext;
    irg = irgn;
  }
}

static int sf_emit_o(sf_run *q, rng_t *r, orc_phot *p, int *irg) {
  const orc_model *m = q->s.m;
  const int nc = q->nc;
  for (int tries = 0; tries < 1000; ++tries) {
    p->pol = 0;
    double Er = q->Etot * rnd(r);
    if (Er < q->Estar) {
      p->E = q->Etot;
      p->scatt = 0;
      if (sf_star_start_o(q, r, p, irg, 0)) return 1;
      continue;
    }
    p->scatt = 1;
    Er = Er - q->Estar;
    long k = 0; /* the cell scan of TraceMono.f:1253-1256 */
    while (k < q->ncum && !(Er < q->cum[k])) ++k;
    if (k >= q->ncum) continue;
    const int i = 1 + (int)(k / nc), j = 1 + (int)(k % nc);
    double Rad = rnd(r);
    Rad = sqrt(m->R[i] * m->R[i] * Rad + m->R[i + 1] * m->R[i + 1] * (1.0 - Rad));
    double Th = rnd(r);
    Th = m->Theta[j - 1] * Th + m->Theta[j] * (1.0 - Th);
    p->z = Rad * Th;
    if (rnd(r) < 0.5) p->z = -p->z;
    const double phi = (rnd(r) * PI_D) * 2.0;
    p->x = (Rad * sqrt(1.0 - Th * Th)) * dm_sin(phi);
    p->y = (Rad * sqrt(1.0 - Th * Th)) * dm_cos(phi);
    randomdirection(r, &p->vx, &p->vy, &p->vz);
    p->i = i;
    p->j = j;
    *irg = sub_irg(&q->g, j, acos(fabs(p->z) / sqrt((p->x * p->x + p->y * p->y) + p->z * p->z)));
    p->onEdge = 0;
    p->edgeNr = 0;
    p->E = q->Etot / q->vis[(size_t)i * nc + (j - 1)];
    return 1;
  }
  return 0;
}

static void sf_mc_packet(sf_run *q, uint64_t key, int64_t w) {
  const orc_model *m = q->s.m;
  const int nc = q->nc;
  rng_t r;
  memset(&r, 0, sizeof r);
  px_init(&r.px, key, (uint64_t)(q->nstar + w));
  orc_phot p;
  memset(&p, 0, sizeof p);
  int irg = 1, ia[SF_NPHI_O];
  double Qd[SF_NPHI_O];
  if (!sf_emit_o(q, &r, &p, &irg)) {
    q->info[3]++;
    return;
  }
  p.E = p.E / (double)(float)q->nphot;
  if (q->mode == 2) {
    p.pol = 0;
    p.Q = p.U = p.V = 0.0;
    double x = 1.0, y = 0.0, z = 0.0;
    if (p.vz != 1.0) {
      x = -p.vy;
      y = p.vx;
    }
    const double rr = sqrt((x * x + y * y) + z * z);
    p.Sx = x / rr;
    p.Sy = y / rr;
    p.Sz = z / rr;
  }
  const int maxv = (m->nr + m->nt + 360) * 2;
  for (int nint = 0;; ++nint) {
    const double tau0 = -dm_log(rnd(&r));
    if (q->mode == 2 && p.scatt) sf_dirs_o(q, &p, ia, Qd);
    double tau = 0.0;
    int escape = 0, interact = 0;
    for (int nv = 1;; ++nv) {
      double v;
      int inext, jnext, irgn;
      if (nv > maxv) {
        escape = 1;
        break;
      }
      if (trace2edge_rg(&q->s, &q->g, &p, irg, &v, &inext, &jnext, &irgn) != 0) {
        q->info[1]++;
        escape = 1;
        break;
      }
      const size_t c = (size_t)p.i * nc + (p.j - 1);
      const double tau1 = ((v * m->dens[c]) * q->kext[c]) * AU_CM;
      if (tau + tau1 > tau0) {
        v = (v * (tau0 - tau)) / tau1;
        interact = 1;
      }
      if (p.scatt) {
        if (q->mode == 1) {
          const size_t b = sf_base_o(q, p.i, p.j, 1, 0);
          q->SF[b] = q->SF[b] + ((p.E * v) * AU_CM) / 2.0;
          q->SF[b + SF_NB_O] = q->SF[b + SF_NB_O] + ((p.E * v) * AU_CM) / 2.0;
        } else {
          const double x = p.x + (p.vx * v) / 2.0, y = p.y + (p.vy * v) / 2.0;
          const size_t b = sf_base_o(q, p.i, p.j, irg < 1 ? 1 : irg, p.z > 0.0 ? 0 : 1);
          q->SF[b] = q->SF[b] + (p.E * v) * AU_CM;
          sf_fold_o(q, b, q->F + c * 1082, x, y, p.E, (v * AU_CM) / 2.0, ia, Qd, 1);
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
      if (inext >= m->nr || inext < 0) {
        escape = 1;
        break;
      }
      p.i = inext;
      p.j = jnext;
      irg = irgn;
    }
    if (escape) return;
    const size_t c = (size_t)p.i * nc + (p.j - 1);
    const double alb = q->alb[c];
    const double fstop = sqrt(sqrt(alb));
    if (!(fstop > 0.0)) return;
    const double fact = alb / fstop;
    p.E = p.E * fact;
    p.Q = p.Q * fact;
    p.U = p.U * fact;
    p.V = p.V * fact;
    if (rnd(&r) > fstop) return;
    if (nint >= 1000000) {
      q->info[2]++;
      return;
    }
    p.scatt = 1;
    if (q->mode == 1)
      randomdirection(&r, &p.vx, &p.vy, &p.vz);
    else
      scatangle(&q->s, &r, &p, q->F + c * 1082, q->F + c * 1082 + 1080);
  }
}

int orc_scatter_field(const orc_model *m, const double *Kabs_c, const double *Ksca_c, const double *T, int scat_how,
                      double angle, double lam0, int64_t nphot, int64_t nstar, uint64_t key, int nexits, double *SF,
                      int64_t *info) {
  const int nR = m->nr, nt = m->nt, nc = nt - 1, ncell = nR * nc, nlam = m->nlam, TT = ORC_TMAX + 1;
  sf_run q;
  memset(&q, 0, sizeof q);
  q.s.m = m;
  q.s.nc = nc;
  q.s.scat_how = scat_how;
  q.nc = nc;
  q.mode = scat_how == 2 ? 2 : 1;
  q.nstar = nstar;
  q.nphot = nphot;
  q.info = info;
  q.SF = SF;
  for (int k = 0; k < 4; ++k) info[k] = 0;
  sub_build(m, q.mode == 2, &q.g);
  info[0] = q.g.nsub;
  /* the wavelength bracket of TraceMono.f:617-643 */
  int l1 = 0, l2 = 1;
  double w1 = 1.0, w2 = 0.0;
  for (int i = 0; i < nlam - 1; ++i)
    if (lam0 >= m->lam[i] && lam0 <= m->lam[i + 1]) {
      l1 = i;
      l2 = i + 1;
      w1 = (m->lam[i + 1] - lam0) / (m->lam[i + 1] - m->lam[i]);
      w2 = (lam0 - m->lam[i]) / (m->lam[i + 1] - m->lam[i]);
    }
  if (lam0 >= m->lam[nlam - 1]) {
    l1 = nlam - 2;
    l2 = nlam - 1;
    w1 = 0.0;
    w2 = 1.0;
  }
  q.kabs = (double *)malloc(sizeof(double) * ncell);
  q.kext = (double *)malloc(sizeof(double) * ncell);
  q.alb = (double *)malloc(sizeof(double) * ncell);
  q.vis = (double *)malloc(sizeof(double) * ncell);
  double *emis = (double *)calloc((size_t)ncell, sizeof(double)), *ksca = (double *)malloc(sizeof(double) * ncell);
  if (q.mode == 2) q.F = (double *)malloc(sizeof(double) * (size_t)ncell * 1082);
  for (int c = 0; c < ncell; ++c) {
    const double *w = m->comp_w + (size_t)c * m->ncomp;
    double Ka = 0.0, Ke = 0.0, Ks = 0.0;
    for (int k = 0; k < m->ncomp; ++k) {
      const double *a = Kabs_c + (size_t)k * nlam, *s = Ksca_c + (size_t)k * nlam;
      Ka = Ka + (w1 * a[l1] + w2 * a[l2]) * w[k];
      Ke = Ke + (w1 * (a[l1] + s[l1]) + w2 * (a[l2] + s[l2])) * w[k];
      Ks = Ks + (w1 * s[l1] + w2 * s[l2]) * w[k];
    }
    q.kabs[c] = Ka;
    q.kext[c] = Ke;
    ksca[c] = Ks;
    q.alb[c] = Ks / Ke;
    if (q.mode == 2)
      for (int e = 0; e < 1082; ++e) {
        double f;
        if (Ks == 0.0) {
          f = e < 180 ? 1.0 : 0.0;
        } else {
          f = 0.0;
          for (int k = 0; k < m->ncomp; ++k) {
            const double *ks = Ksca_c + (size_t)k * nlam;
            double f1, f2;
            if (e < 1080) {
              f1 = m->F_comp[((size_t)k * nlam + l1) * 1080 + e];
              f2 = m->F_comp[((size_t)k * nlam + l2) * 1080 + e];
            } else {
              f1 = m->IF_comp[((size_t)k * nlam + l1) * 2 + (e - 1080)];
              f2 = m->IF_comp[((size_t)k * nlam + l2) * 2 + (e - 1080)];
            }
            f = f + ((f1 * ks[l1]) * w1 + (f2 * ks[l2]) * w2) * w[k];
          }
          f = f / Ks;
        }
        q.F[(size_t)c * 1082 + e] = f;
      }
  }
  /* EmissionDistribution: the thermal weight, the exit depth and the running sum */
  q.ncum = (long)(nR - 1) * nc;
  q.cum = (double *)malloc(sizeof(double) * (q.ncum > 0 ? q.ncum : 1));
  double Et = 0.0;
  for (int i = 1; i <= nR - 1; ++i)
    for (int j = 1; j <= nc; ++j) {
      const int c = i * nc + (j - 1);
      double e = 0.0;
      if (T[c] != 0.0) {
        int iT = (int)(T[c] / 1.0);
        const double wT1 = (double)(iT + 1) - T[c] / 1.0, wT2 = T[c] / 1.0 - (double)iT;
        if (iT < 1) iT = 1;
        if (iT > ORC_TMAX - 1) iT = ORC_TMAX - 1;
        const double *w = m->comp_w + (size_t)c * m->ncomp;
        const double *B1 = m->BB + (size_t)l1 * TT, *B2 = m->BB + (size_t)l2 * TT;
        for (int k = 0; k < m->ncomp; ++k) {
          const double *a = Kabs_c + (size_t)k * nlam;
          e = e + ((w1 * (wT1 * B1[iT] + wT2 * B1[iT + 1])) * a[l1] + (w2 * (wT1 * B2[iT] + wT2 * B2[iT + 1])) * a[l2]) *
                      w[k];
        }
      }
      e = (e * m->dens[c]) * m->V[c];
      double taumin = 0.0;
      for (int k = 1; k <= nexits; ++k) {
        orc_phot p;
        memset(&p, 0, sizeof p);
        double Rad = 0.5;
        Rad = sqrt(m->R[i] * m->R[i] * Rad + m->R[i + 1] * m->R[i + 1] * (1.0 - Rad));
        double Th = 0.5;
        Th = m->Theta[j - 1] * Th + m->Theta[j] * (1.0 - Th);
        p.z = Rad * Th;
        double phi = 1e-4;
        p.x = Rad * sqrt(1.0 - Th * Th) * dm_sin(phi);
        p.y = Rad * sqrt(1.0 - Th * Th) * dm_cos(phi);
        phi = (PI_D * (double)(float)(k - 1)) / (double)(float)(nexits - 1);
        p.vy = dm_cos(phi);
        p.vz = dm_sin(phi);
        p.i = i;
        p.j = j;
        p.onEdge = 0;
        double tau = 0.0;
        for (int n = 0; n < 1000000; ++n) {
          double v;
          int inext, jnext;
          if (trace2edge(&q.s, &p, &v, &inext, &jnext) != 0) break;
          p.onEdge = 1;
          p.x = p.x + p.vx * v;
          p.y = p.y + p.vy * v;
          p.z = p.z + p.vz * v;
          const int cc = p.i * nc + (p.j - 1);
          tau = tau + ((v * m->dens[cc]) * AU_CM) * q.kabs[cc];
          if (inext >= nR || inext <= 0) break;
          p.i = inext;
          p.j = jnext;
        }
        if (tau < taumin || k == 1) taumin = tau;
      }
      q.vis[c] = nexits > 0 ? dm_exp(-taumin) : 1.0;
      emis[c] = e * q.vis[c];
      Et = Et + emis[c];
      q.cum[(size_t)(i - 1) * nc + (j - 1)] = Et;
    }
  q.Estar = m->Fstar[l1] * w1 + m->Fstar[l2] * w2;
  q.Etot = Et + q.Estar;
  q.dirs = (double *)calloc(3 * SF_NPHI_O, sizeof(double));
  if (q.mode == 2)
    for (int i = 1; i <= SF_NPHI_O; ++i) { /* TracePath, TraceMono.f:2058-2075 */
      const double phi = (PI_D * ((double)(float)i - 0.5)) / ((double)(float)SF_NPHI_O / 2.0);
      double x = 0.0, y = 0.0, z = 1.0;
      rotate(&x, &y, &z, 0.0, 1.0, 0.0, angle);
      rotate(&x, &y, &z, 0.0, 0.0, 1.0, phi);
      const double r = sqrt((x * x + y * y) + z * z);
      q.dirs[3 * (i - 1)] = x / r;
      q.dirs[3 * (i - 1) + 1] = y / r;
      q.dirs[3 * (i - 1) + 2] = z / r;
    }
  memset(SF, 0, sizeof(double) * (size_t)nR * q.g.nsub * 2 * SF_NB_O);
  for (int64_t w = 0; w < nstar; ++w) sf_star_packet(&q, key, w);
  if (q.Etot > 0.0)
    for (int64_t w = 0; w < nphot; ++w) sf_mc_packet(&q, key, w);
  free(q.kabs); free(q.kext); free(q.alb); free(q.vis); free(emis); free(ksca); free(q.F); free(q.cum); free(q.dirs);
  sub_free(&q.g);
  return 0;
}
