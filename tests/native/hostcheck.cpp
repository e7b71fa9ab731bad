// Host build of the device cores (dhs_core.cuh, transport_core.cuh) for the
// CPU tests: the same source the GPU kernels run, executed by one host
// thread, so it can be compared bit for bit with the oracle without a GPU.
// Test infrastructure only.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../mcmax_b200/csrc/dhs_core.cuh"
#include "../../mcmax_b200/csrc/transport_core.cuh"
#include "../../mcmax_b200/csrc/diffuse_core.cuh"
#include "../../mcmax_b200/csrc/dstruct_core.cuh"
#include "../../mcmax_b200/csrc/rt_core.cuh"
#include "../../mcmax_b200/csrc/surrogate_phase.h"

extern "C" {

int hc_dhs_sample(double rcore, double rshell, double wvno, double mre, double mim, const double *mu, double *F,
                  double *ce, double *cs) {
  int n1 = dhs_nmx1(rshell, wvno, mre, -mim);
  if (n1 > 300000) n1 = 300000;
  std::vector<cx> scratch(4 * (size_t)(n1 + 2));
  return dhs_sample<1, 90>(rcore, rshell, wvno, mre, -mim, mu, scratch.data(), n1 + 2, 0, F, F + 180, F + 360,
                           F + 540, ce, cs);
}

int hc_mie_sample(double rad, double lam, double e1, double e2, double *F, double *cs, double *ce) {
  int nmax, nfi, nD;
  mie_counts(rad, lam, e1, e2, &nmax, &nfi, &nD);
  int cap = (nfi > nD ? nfi : nD) + 2;
  std::vector<double> scratch(8 * (size_t)cap);
  return mie_sample<1, 90>(rad, lam, e1, e2, scratch.data(), cap, 0, F, F + 180, F + 360, F + 540, cs, ce);
}

struct HcModel {
  int nr, nt, nlam, ncomp, scat_how, uniform_mix, rw;
  double factRW, Lstar;
  int64_t nphot, maxinteract;
  uint64_t seed;
  const double *R, *Theta, *SinTheta, *dens, *V, *nu, *BB, *Fstar;
  const double *KabsTot, *KscaTot, *KpCell, *comp_w, *Ksca_c, *F_c, *IF_c;
  const double *sinthet, *cos2phi, *sin2phi, *KDext, *KDabs, *rw_y, *rw_phi;
  const unsigned char *thick;
};

// serial run of the device packet loop on the host; outputs as the oracle's
int hc_mcradiation(const HcModel *h, double *EJv, double *EJv2, double *Eabs, double *T, int *Ni, double *spec,
                   double *scatspec, int *ispec, unsigned long long *counters, double *tautot) {
  const int nc = h->nt - 1, ncell = h->nr * nc, nlam = h->nlam;
  std::vector<double> dens(ncell), mass(ncell), dnu_half(nlam - 1), star_cdf(nlam - 1), wlam(nlam);
  for (int c = 0; c < ncell; ++c) {
    mass[c] = h->dens[c] * h->V[c];
    dens[c] = h->dens[c] <= 1e-50 ? 1e-50 : h->dens[c];
  }
  for (int i = 0; i < nlam - 1; ++i) dnu_half[i] = std::fabs(h->nu[i] - h->nu[i + 1]) * 0.5;
  double Lt = 0.0;
  for (int i = 0; i < nlam - 1; ++i) {
    Lt = Lt + dnu_half[i] * (h->Fstar[i] + h->Fstar[i + 1]);
    star_cdf[i] = Lt;
  }
  for (int i = 0; i < nlam; ++i) {
    if (i == 0)
      wlam[i] = -1e23 / (h->nu[1] / 2.0);
    else if (i == nlam - 1)
      wlam[i] = -1e23 / ((h->nu[nlam - 1] - h->nu[nlam - 2]) / 2.0);
    else
      wlam[i] = -1e23 / ((h->nu[i + 1] - h->nu[i - 1]) / 2.0);
  }
  std::vector<double> emit_cdf;
  if (h->uniform_mix) {
    emit_cdf.resize((size_t)TP_TMAX * (nlam - 1));
    for (int iT = 0; iT < TP_TMAX; ++iT) {
      double L = 0.0, s0 = (h->BB[iT + 1] - h->BB[iT]) * h->KabsTot[0];
      for (int i = 0; i < nlam - 1; ++i) {
        const double *B = h->BB + (size_t)(i + 1) * TP_TT;
        double s1 = (B[iT + 1] - B[iT]) * h->KabsTot[i + 1];
        L = L + dnu_half[i] * (s0 + s1);
        emit_cdf[(size_t)iT * (nlam - 1) + i] = L;
        s0 = s1;
      }
    }
  }
  std::vector<int> kd_index(ncell, -1);
  for (int c = 0; c < ncell; ++c)
    if (h->thick && h->thick[c]) kd_index[c] = c;
  TModel m;
  memset(&m, 0, sizeof m);
  m.nr = h->nr; m.nt = h->nt; m.nc = nc; m.ncell = ncell; m.nlam = nlam; m.ncomp = h->ncomp;
  m.scat_how = h->scat_how;
  m.scattering = 0;
  if (h->scat_how != 0)
    for (size_t k = 0; k < (size_t)ncell * nlam; ++k)
      if (h->KscaTot[k] != 0.0) { m.scattering = 1; break; }
  m.uniform_mix = h->uniform_mix;
  m.rw = h->rw;
  m.factRW = h->factRW;
  m.R0 = h->R[0];
  m.Lstar = h->Lstar;
  m.Epkt = h->Lstar / ((double)h->nphot * 1.0);
  m.nphot = h->nphot;
  m.maxinteract = h->maxinteract;
  m.pid0 = 0;
  m.nruns_d = 1.0;
  m.seed = h->seed;
  m.R = h->R; m.Theta = h->Theta; m.SinTheta = h->SinTheta; m.dens = dens.data(); m.mass = mass.data();
  m.nu = h->nu; m.dnu_half = dnu_half.data(); m.BB = h->BB; m.star_cdf = star_cdf.data(); m.wlam = wlam.data();
  m.KabsTot = h->KabsTot; m.KscaTot = h->KscaTot; m.KpCell = h->KpCell;
  m.emit_cdf = h->uniform_mix ? emit_cdf.data() : nullptr;
  m.comp_w = h->comp_w; m.Ksca_c = h->Ksca_c; m.F_c = h->F_c; m.IF_c = h->IF_c;
  m.sinthet = h->sinthet; m.cos2phi = h->cos2phi; m.sin2phi = h->sin2phi;
  m.KDext = h->KDext; m.KDabs = h->KDabs; m.rw_y = h->rw_y; m.rw_phi = h->rw_phi;
  m.kd_index = kd_index.data();
  m.thick = h->thick;
  std::vector<unsigned char> nothick;
  if (!m.thick) {
    nothick.assign(ncell, 0);
    m.thick = nothick.data();
  }
  std::vector<int> lastphot(ncell, 0), kp_hint(ncell, 0);
  unsigned long long next = 0, done = 0, tmark[8] = {0};
  TAcc A;
  memset(&A, 0, sizeof A);
  A.kp_hint = kp_hint.data();
  A.run_packets = h->nphot;
  A.ncell = ncell;
  A.done = &done;
  A.tmark = tmark;
  A.EJv = EJv; A.EJv2 = EJv2; A.Eabs = Eabs; A.T = T; A.Ni = Ni; A.lastphot = lastphot.data();
  A.spec = spec; A.scatspec = scatspec; A.ispec = ispec; A.counters = counters; A.tautot = tautot; A.next = &next;
  TLocal L;
  memset(&L, 0, sizeof L);
  // with uniform_mix the KpCell table has a single row
  if (h->uniform_mix) m.KpCell = h->KpCell;
  for (int64_t pid = 0; pid < h->nphot; ++pid) tp_run_packet(m, A, pid, L);
  for (int k = 0; k < TC_N; ++k) counters[k] += (unsigned long long)L.cnt[k];
  *tautot += L.tautot;
  return 0;
}
}

extern "C" {
void hc_detmath(int which, int n, const double *x, double *y) {
  for (int i = 0; i < n; ++i) {
    switch (which) {
      case 0: y[i] = dm_exp(x[i]); break;
      case 1: y[i] = dm_log(x[i]); break;
      case 2: y[i] = dm_sin(x[i]); break;
      default: y[i] = dm_cos(x[i]); break;
    }
  }
}

void hc_philox(const uint32_t *ctr, const uint32_t *key, uint32_t *out) { px_philox4x32_10(ctr, key, out); }

double hc_tinv(const double *kp, double E1, int lo) {
  int ib;
  return tp_tinv(kp, E1, lo, &ib);
}
}

// ---------------------------------------------------------------------------
// host build of the GPU-ordered kernel (transport_fast.cuh) with host-built
// tables identical to the device table builders
#include "../../mcmax_b200/csrc/transport_fast.cuh"

template <class R>
static int hc_fast_impl(const HcModel *h, double *EJv, double *EJv2, double *Eabs, double *T, int *Ni,
                        double *spec, unsigned long long *counters, double *tautot, int64_t first, int64_t count,
                        int inflight = 1, int *Nabs = nullptr) {
  const int nc = h->nt - 1, ncell = h->nr * nc, nlam = h->nlam, n = nlam - 1, ncomp = h->ncomp;
  std::vector<double> dens(ncell), mass(ncell), dnu(n), star_cdf(n), wlam(nlam);
  for (int c = 0; c < ncell; ++c) {
    mass[c] = h->dens[c] * h->V[c];
    dens[c] = h->dens[c] <= 1e-50 ? 1e-50 : h->dens[c];
  }
  for (int i = 0; i < n; ++i) dnu[i] = std::fabs(h->nu[i] - h->nu[i + 1]) * 0.5;
  double Lt = 0.0;
  for (int i = 0; i < n; ++i) {
    Lt = Lt + dnu[i] * (h->Fstar[i] + h->Fstar[i + 1]);
    star_cdf[i] = Lt;
  }
  for (int i = 0; i < nlam; ++i)
    wlam[i] = i == 0 ? -1e23 / (h->nu[1] / 2.0)
                     : (i == nlam - 1 ? -1e23 / ((h->nu[nlam - 1] - h->nu[nlam - 2]) / 2.0)
                                      : -1e23 / ((h->nu[i + 1] - h->nu[i - 1]) / 2.0));
  const double *K = h->KabsTot;
  std::vector<double> C((size_t)TP_TT * n), D((size_t)TP_TMAX * n);
  for (int iT = 0; iT <= TP_TMAX; ++iT) {
    double L = 0.0, s0 = h->BB[iT] * K[0];
    for (int i = 0; i < n; ++i) {
      double s1 = h->BB[(size_t)(i + 1) * TP_TT + iT] * K[i + 1];
      L = L + dnu[i] * (s0 + s1);
      C[(size_t)iT * n + i] = L;
      s0 = s1;
    }
  }
  for (int iT = 0; iT < TP_TMAX; ++iT) {
    double L = 0.0, s0 = (h->BB[iT + 1] - h->BB[iT]) * K[0];
    for (int i = 0; i < n; ++i) {
      const double *B = h->BB + (size_t)(i + 1) * TP_TT;
      double s1 = (B[iT + 1] - B[iT]) * K[i + 1];
      L = L + dnu[i] * (s0 + s1);
      D[(size_t)iT * n + i] = L;
      s0 = s1;
    }
  }
  std::vector<unsigned short> eG((size_t)TP_TMAX * F_NGUIDE);
  for (int iT = 0; iT < TP_TMAX; ++iT) {
    const double *row = &D[(size_t)iT * n];
    int i = 0;
    for (int g = 0; g < F_NGUIDE; ++g) {
      const double v = row[n - 1] * (double)g / (double)F_NGUIDE;
      while (i < n - 1 && !(row[i] >= v)) ++i;
      eG[(size_t)iT * F_NGUIDE + g] = (unsigned short)i;
    }
  }
  const int nmat = ncomp * nlam;
  std::vector<R> A((size_t)nmat * 180), B((size_t)nmat * 180), F6((size_t)nmat * 1080);
  std::vector<unsigned char> sG((size_t)nmat * F_NGUIDE);
  for (int k = 0; k < nmat; ++k) {
    const double *F11 = h->F_c + (size_t)k * 1080, *F12 = F11 + 180;
    double a = 0.0, b = 0.0;
    for (int j = 0; j < 180; ++j) {
      a += (TP_PI * h->sinthet[j]) * F11[j];
      b += (TP_PI * h->sinthet[j]) * F12[j];
      A[(size_t)k * 180 + j] = (R)a;
      B[(size_t)k * 180 + j] = (R)b;
    }
    for (int e = 0; e < 1080; ++e) F6[(size_t)k * 1080 + e] = (R)h->F_c[(size_t)k * 1080 + e];
    int i = 0;
    for (int g = 0; g < F_NGUIDE; ++g) {
      const R v = A[(size_t)k * 180 + 179] * (R)g / (R)F_NGUIDE;
      while (i < 179 && !(A[(size_t)k * 180 + i] > v)) ++i;
      sG[(size_t)k * F_NGUIDE + g] = (unsigned char)i;
    }
  }
  std::vector<double> c2(181), s2(181), ly(TP_NY);
  c2[0] = s2[0] = 0.0;
  for (int k = 1; k <= 180; ++k) {
    c2[k] = c2[k - 1] + h->cos2phi[k];
    s2[k] = s2[k - 1] + h->sin2phi[k];
  }
  for (int i = 0; i < TP_NY; ++i) ly[i] = std::log(h->rw_y[i]);
  std::vector<R> KaR(nlam), KeR(nlam), KsR((size_t)nmat);
  for (int l = 0; l < nlam; ++l) {
    KaR[l] = (R)h->KabsTot[l];
    KeR[l] = (R)(h->KabsTot[l] + h->KscaTot[l]);
  }
  for (int k = 0; k < nmat; ++k) KsR[k] = (R)h->Ksca_c[k];
  std::vector<int> kd_index(ncell, -1);
  for (int c = 0; c < ncell; ++c)
    if (h->thick && h->thick[c]) kd_index[c] = c;
  std::vector<unsigned char> nothick(ncell, 0);
  FModel<R> m;
  memset(&m, 0, sizeof m);
  m.nr = h->nr; m.nt = h->nt; m.nc = nc; m.ncell = ncell; m.nlam = nlam; m.ncomp = ncomp;
  m.scat_how = h->scat_how;
  for (size_t k = 0; k < (size_t)nlam && h->scat_how; ++k)
    if (h->KscaTot[k] != 0.0) m.scattering = 1;
  m.uniform_mix = 1;
  m.rw = h->rw;
  m.factRW = h->factRW;
  m.R0 = h->R[0];
  m.Lstar = h->Lstar;
  m.Epkt = h->Lstar / ((double)h->nphot * 1.0);
  m.nruns_d = 1.0;
  m.nphot = h->nphot;
  m.maxinteract = h->maxinteract;
  m.seed = h->seed;
  m.Rr = h->R; m.Theta = h->Theta; m.SinTheta = h->SinTheta; m.star_cdf = star_cdf.data();
  m.KabsRow = KaR.data(); m.KextRow = KeR.data(); m.Ksca_c = KsR.data();
  m.c2cum = c2.data(); m.s2cum = s2.data();
  m.dens = dens.data(); m.mass = mass.data(); m.wlam = wlam.data();
  m.KabsTot = h->KabsTot; m.BB = h->BB; m.dnu_half = dnu.data(); m.KpCell = h->KpCell;
  m.Ccum = C.data(); m.Dcum = D.data(); m.comp_w = h->comp_w;
  m.scatA = A.data(); m.scatB = B.data(); m.F6 = F6.data(); m.IF_c = h->IF_c;
  m.scatG = sG.data(); m.emitG = eG.data();
  m.KDext = h->KDext; m.KDabs = h->KDabs; m.rw_logy = ly.data(); m.rw_phi = h->rw_phi;
  m.kd_index = kd_index.data(); m.thick = h->thick ? h->thick : nothick.data();
  std::vector<int> lastphot(ncell, 0), kp_hint(ncell, 0), ispec((size_t)nlam * 31, 0);
  std::vector<double> scatspec((size_t)nlam * 31, 0.0);
  unsigned long long next = 0, done = 0, tmark[8] = {0};
  TAcc Ac;
  memset(&Ac, 0, sizeof Ac);
  Ac.EJv = EJv; Ac.EJv2 = EJv2; Ac.Eabs = Eabs; Ac.T = T; Ac.Ni = Ni; Ac.lastphot = lastphot.data();
  Ac.kp_hint = kp_hint.data(); Ac.spec = spec; Ac.scatspec = scatspec.data(); Ac.ispec = ispec.data();
  Ac.counters = counters; Ac.tautot = tautot; Ac.next = &next; Ac.run_packets = h->nphot; Ac.ncell = ncell;
  Ac.done = &done; Ac.tmark = tmark;
  Ac.Nabs = Nabs;
  TLocal L;
  memset(&L, 0, sizeof L);
  if (inflight <= 1) {
    for (int64_t pid = first; pid < first + count; ++pid) f_run_packet<R>(m, Ac, pid, L);
  } else {
    /* `inflight` packets at once, each advanced by one event in turn: the
     * cell energies a packet sees include the deposits of packets started
     * after it, as on the GPU */
    std::vector<FSlot<R>> slots(inflight);
    std::vector<char> live(inflight, 0);
    int64_t next_pid = first;
    const int64_t end = first + count;
    int nlive = 0;
    for (int k = 0; k < inflight && next_pid < end; ++k, ++nlive) {
      f_slot_start<R>(m, Ac, slots[k], next_pid++);
      live[k] = 1;
    }
    while (nlive > 0) {
      for (int k = 0; k < inflight; ++k) {
        if (!live[k]) continue;
        if (f_slot_step<R>(m, Ac, slots[k], L)) {
          if (next_pid < end) {
            f_slot_start<R>(m, Ac, slots[k], next_pid++);
          } else {
            live[k] = 0;
            --nlive;
          }
        }
      }
    }
  }
  for (int k = 0; k < TC_N; ++k) counters[k] += (unsigned long long)L.cnt[k];
  *tautot += L.tautot;
  return 0;
}

extern "C" int hc_fast(const HcModel *h, int mixed, double *EJv, double *EJv2, double *Eabs, double *T, int *Ni,
                       double *spec, unsigned long long *counters, double *tautot, int64_t first, int64_t count) {
  if (mixed) return hc_fast_impl<float>(h, EJv, EJv2, Eabs, T, Ni, spec, counters, tautot, first, count);
  return hc_fast_impl<double>(h, EJv, EJv2, Eabs, T, Ni, spec, counters, tautot, first, count);
}

/* the GPU-ordered kernel with `inflight` packets interleaved event by event
 * (the concurrency of a device launch, emulated in one host thread); Nabs
 * per cell */
extern "C" int hc_fast_interleaved(const HcModel *h, int mixed, double *EJv, double *EJv2, double *Eabs, double *T,
                                   int *Ni, double *spec, unsigned long long *counters, double *tautot,
                                   int inflight, int *Nabs) {
  if (mixed)
    return hc_fast_impl<float>(h, EJv, EJv2, Eabs, T, Ni, spec, counters, tautot, 0, h->nphot, inflight, Nabs);
  return hc_fast_impl<double>(h, EJv, EJv2, Eabs, T, Ni, spec, counters, tautot, 0, h->nphot, inflight, Nabs);
}

/* Diffuse on the host: the host logic of mcg_diffuse with a backend of
 * serial loops over the kernels' per-element functions */
struct HcDiffuseTables {
  int nlam, ncomp, scattering, uniform_mix;
  const double *comp_w, *g_c, *Ksca_c, *KabsTot, *KscaTot, *nu, *BB, *KpCell;
};

struct HostDiffuseBackend {
  const HcDiffuseTables *t;
  std::vector<double> dnu_half;
  bool kd(int n, const int *cells, const int *iTs, double *out) {
    for (int k = 0; k < n; ++k)
      out[k] = df_kd_ext(cells[k], iTs[k], t->nlam, t->ncomp, t->scattering, t->comp_w, t->g_c, t->Ksca_c,
                         t->KabsTot, t->KscaTot, dnu_half.data(), t->BB);
    return true;
  }
  bool kp(int n, const int *cells, const int *iTs, double *out) {
    for (int k = 0; k < n; ++k) out[k] = t->KpCell[(t->uniform_mix ? (size_t)0 : (size_t)cells[k] * DF_TT) + iTs[k]];
    return true;
  }
  bool solve(int nb, int w, const double *coef, const double *rhs, double *x, int *code) {
    *code = df_band_solve_host(nb, w, coef, rhs, x);
    return true;
  }
};

extern "C" int hc_diffuse(int nr, int nt, const double *R, const double *Theta, const double *dens_in,
                          const HcDiffuseTables *t, int nphotmin, double dtmax, double factRW, const int *Ni,
                          const double *dT, double *T, double *EJv, int *stats) {
  const int ncell = nr * (nt - 1);
  std::vector<double> dens(ncell);
  for (int c = 0; c < ncell; ++c) dens[c] = dens_in[c] <= 1e-50 ? 1e-50 : dens_in[c];
  HostDiffuseBackend be;
  be.t = t;
  be.dnu_half.resize(t->nlam > 1 ? t->nlam - 1 : 1);
  for (int i = 0; i < t->nlam - 1; ++i) be.dnu_half[i] = std::fabs(t->nu[i] - t->nu[i + 1]) * 0.5;
  DfGrid g{nr, nt, R, Theta, dens.data(), t->ncomp, t->comp_w};
  DfStats st;
  df_diffuse(g, be, nphotmin, dtmax, factRW, (const int32_t *)Ni, dT, T, EJv, &st);
  stats[0] = st.ncor;
  stats[1] = st.nunknown;
  stats[2] = st.nsolved;
  stats[3] = st.failed;
  stats[4] = st.nb;
  stats[5] = st.w;
  return 0;
}

/* the band solve alone: coef nb*5 stencil slots, rhs nb -> x nb; returns
 * 0 or 1 + the first step with a zero or non-finite pivot */
extern "C" int hc_band_solve(int nb, int w, const double *coef, const double *rhs, double *x) {
  return df_band_solve_host(nb, w, coef, rhs, x);
}

/* DiskStructure on the host: the host logic of mcg_disk_structure with its
 * kernels replaced by serial loops over the same per-column and per-cell
 * functions.  zones as orc_disk_structure (7 values each); shtype: ng
 * scale-height types or NULL. */
struct HostStructBackend {
  bool columns(const DsGrid &g, const DsTables &t, const double *Temp, int ncol, const DsColumn *cols,
               const int *ring, const std::vector<double> &prof, double *rho) {
    ds_columns_host(g, t, Temp, ncol, cols, ring, prof, rho);
    return true;
  }
  bool cells(const DsGrid &g, const double *rho, double *dens, double *dens0, double *gasdens, double *w,
             double *w0) {
    ds_cells_host(g, rho, dens, dens0, gasdens, w, w0);
    return true;
  }
};

extern "C" int hc_disk_structure(int nR, int nTheta, int ng, const double *R, const double *Theta, const double *V,
                                 double Mstar, int nzones, const double *zones, const double *shscale,
                                 const double *grain_scale, const int *shtype, const double *Temp, double *dens,
                                 double *dens0, double *gasdens, double *w, double *w0) {
  std::vector<DsZone> zs(nzones > 0 ? nzones : 0);
  for (int k = 0; k < nzones; ++k) {
    const double *z = zones + 7 * k;
    zs[k] = DsZone{z[0], z[1], z[2], z[3], z[4], z[5], z[6] != 0.0};
  }
  DsGrid g{nR, nTheta, ng, R, Theta, V, Mstar, nzones, zs.data(), shscale, grain_scale, shtype};
  HostStructBackend be;
  return ds_disk_structure(g, be, Temp, dens, dens0, gasdens, w, w0) ? 0 : 1;
}

/* the ray-traced spectrum on the host: the host logic of
 * mcg_trace_spectrum with its kernels replaced by loops over rt_cell and
 * rt_ray.  dens is used as given (the library floors it at 1e-50). */
struct HostRtBackend {
  TModel m;
  int ncomp, nlam;
  const double *comp_w, *Kabs_c, *Ksca_c, *BB, *lam, *T, *dens;
  std::vector<double> kext, emis;
  bool cells(double lam0, double *kx, double *em) {
    int l1, l2;
    double w1, w2;
    rt_lam(nlam, lam, lam0, &l1, &l2, &w1, &w2);
    const int ncell = m.nr * (m.nt - 1);
    kext.resize(ncell);
    emis.resize(ncell);
    for (int c = 0; c < ncell; ++c)
      rt_cell(c, ncomp, nlam, comp_w, Kabs_c, Ksca_c, BB, T[c], l1, l2, w1, w2, &kext[c], &emis[c]);
    std::copy(kext.begin(), kext.end(), kx);
    std::copy(emis.begin(), emis.end(), em);
    return true;
  }
  bool field(double) { return true; } /* the host replay has no scattered-light field */
  bool rays(const std::vector<double> &R, const std::vector<double> &phi, double fstar, const RtOptions &o,
            double *image, int *bad) {
    const int nr = (int)R.size(), nphi = (int)phi.size();
    *bad = 0;
    for (int i = 0; i < nr; ++i)
      for (int k = 0; k < nphi; ++k) {
        int steps;
        image[(size_t)i * nphi + k] = rt_ray(m, dens, kext.data(), emis.data(), R[i], phi[k], o.angle, fstar,
                                              o.dimstar, o.tracestar, 1 << 20, &steps);
        if (steps < 0) ++*bad;
      }
    return true;
  }
};

extern "C" int hc_trace_spectrum(int nr, int nt, const double *R, const double *Theta, const double *dens,
                                 int scat_how, int ncomp, int nlam, const double *comp_w, const double *Kabs_c,
                                 const double *Ksca_c, const double *BB, const double *lam, const double *Fstar,
                                 const double *T, double angle, int nphi, int nj0, int nRfix, const double *Rfix,
                                 double lam_path, int tracestar, double dimstar, int nobs, const double *lam_obs,
                                 double *flux, int *info, double *Rimg_out, int Rimg_cap, double *image_out) {
  TModel m;
  memset(&m, 0, sizeof m);
  m.nr = nr;
  m.nt = nt;
  m.nc = nt - 1;
  m.ncell = nr * (nt - 1);
  m.scat_how = scat_how;
  m.R = R;
  m.Theta = Theta;
  HostRtBackend be;
  be.m = m;
  be.ncomp = ncomp;
  be.nlam = nlam;
  be.comp_w = comp_w;
  be.Kabs_c = Kabs_c;
  be.Ksca_c = Ksca_c;
  be.BB = BB;
  be.lam = lam;
  be.T = T;
  be.dens = dens;
  RtOptions o{angle, nphi, nj0, nRfix, Rfix, lam_path, tracestar, dimstar};
  std::vector<double> Rimg, image;
  int bad = 0;
  if (!rt_spectrum(m, be, o, nlam, lam, Fstar, dens, nobs, lam_obs, flux, &Rimg, &image, &bad)) return 1;
  info[0] = (int)Rimg.size();
  info[1] = bad;
  for (int i = 0; i < (int)Rimg.size() && i < Rimg_cap; ++i) Rimg_out[i] = Rimg[i];
  if (image_out && (int)Rimg.size() <= Rimg_cap)
    std::copy(image.begin(), image.end(), image_out);
  return 0;
}

/* the rectangular image on the host: mcg_trace_image's host logic with the
 * sample and pixel kernels replaced by one loop over the points in order */
extern "C" int hc_trace_image(int nr, int nt, const double *R, const double *Theta, const double *dens, int scat_how,
                              int ncomp, int nlam, const double *comp_w, const double *Kabs_c, const double *Ksca_c,
                              const double *BB, const double *lam, const double *Fstar, const double *T, double angle,
                              int nphi, int nj0, int nRfix, const double *Rfix, int tracestar, double dimstar,
                              double lam0, int npix, int nint, double Rmax, double pa, unsigned long long seed,
                              int linear, double *flux, double *im, int *info) {
  const int cap = (int)rt_image_radii_count(nr, nt, nj0, nRfix, scat_how);
  std::vector<double> Rimg(cap), image((size_t)cap * nphi);
  if (hc_trace_spectrum(nr, nt, R, Theta, dens, scat_how, ncomp, nlam, comp_w, Kabs_c, Ksca_c, BB, lam, Fstar, T,
                        angle, nphi, nj0, nRfix, Rfix, lam0, tracestar, dimstar, 1, &lam0, flux, info, Rimg.data(),
                        cap, image.data()) != 0)
    return 1;
  const int ni = info[0];
  if (ni > cap) return 2;
  std::fill(im, im + (size_t)npix * npix, 0.0);
  const long long ns = (long long)(ni - 1) * nphi * nint;
  for (long long s = 0; s < ns; ++s) {
    uint32_t key[2];
    double v;
    rt_image_sample(s, nphi, nint, Rimg.data(), image.data(), (uint64_t)seed, Rmax, pa, npix, linear, key, &v);
    for (int m = 0; m < 2; ++m)
      if (key[m] < (uint32_t)npix * (uint32_t)npix) im[key[m]] = im[key[m]] + v;
  }
  return 0;
}

/* the surrogate's Mueller matrix F[6][180] from moments [0..12] */
extern "C" void hc_surr_phase(const double *chi, const double *beta, const double *gam, const double *del, int deltam,
                              double *F) {
  static const SurrLegendre legendre;
  surr_phase_matrix(legendre, chi, beta, gam, del, deltam, F);
}
