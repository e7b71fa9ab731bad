/*
 * rt_core.cuh -- ray-traced flux of the disk at one inclination (the
 * 'SPECTRUM' observation of Telescope.f:137-160: TracePath once, then
 * TraceFlux per wavelength), for the thermal emission of the dust and the
 * attenuated star, and with a scattered-light field (scat_core.cuh) its
 * scattered light.
 *
 *   image rays     TracePath (TraceMono.f:2032-2297): radial points from the
 *                  tau = 0.1 radius along the midplane (tau01R,
 *                  TraceMono.f:2300-2345), the fixed radii, nj0 points per
 *                  radial cell, nstar points over the stellar disk, the outer
 *                  edge; nphi angles over half the image plane
 *   ray path       trace2dpath (TraceMono.f:2350-2431) with the packet loop's
 *                  cell-edge geometry (tp_trace2edge; Trace2edgeRG with one
 *                  sub-cell per cell is the same code)
 *   formal solution TraceFlux (TraceMono.f:331-474): emission
 *                  B(T) Kabs/Kext (1 - albedo) per cell plus twice the
 *                  scattered source of the field when there is one
 *                  (sf_segment_source; the path then also carries the
 *                  sub-cell, the folded azimuth bins of its ends and the
 *                  side of the midplane it ends on, and steps with
 *                  Trace2edgeRG), the exp(-tau) attenuation with its
 *                  tau < 1e-6 branch, the star's intensity behind the disk
 *   flux           the trapezoid over image radii and angles (TraceMono.f:
 *                  481-497)
 *
 * Where the reference's tau01R traces with the opacities of the last packet
 * its Monte Carlo emitted (Grain%KextL is not set for that trace), this
 * traces with the opacities at the wavelength TracePath is given (0.55
 * micron for a spectrum); the radius only places image rays.
 *
 * Shared by the library (raytrace.cu: one thread per image ray) and the
 * host replay; every a*b+c is rounded twice and the rotations use detmath.h,
 * so both give the same bits.
 */
#ifndef MCMAX_RT_CORE_CUH
#define MCMAX_RT_CORE_CUH

#include <math.h>
#include <stddef.h>

#include <algorithm>
#include <vector>

#include "scat_core.cuh"
#include "transport_core.cuh"

#ifdef __CUDACC__
#define RT_HD __host__ __device__ inline
#else
#define RT_HD static inline
#endif

#define RT_AU ((double)1.49598e13f)
#define RT_PI 3.14159265358979323846
#define RT_NSTAR 30
#define RT_TAU_MAX 1e8

/* wavelength bracket of lam0 (TraceMono.f:45-63) */
RT_HD void rt_lam(int nlam, const double *lam, double lam0, int *l1, int *l2, double *w1, double *w2) {
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

/* one cell at the wavelength (l1, l2, w1, w2): extinction and the source
 * function emis (TraceMono.f:165-176 and 232-255 for thermal contact).  Kext
 * of a component is Kabs + Ksca. */
RT_HD void rt_cell(int c, int ncomp, int nlam, const double *comp_w, const double *Kabs_c, const double *Ksca_c,
                   const double *BB, double T, int l1, int l2, double w1, double w2, double *kext, double *emis) {
  const double *w = comp_w + (size_t)c * ncomp;
  double Kabs = 0.0, Kext = 0.0, Ksca = 0.0;
  for (int q = 0; q < ncomp; ++q) {
    const double *Ka = Kabs_c + (size_t)q * nlam, *Ks = Ksca_c + (size_t)q * nlam;
    Kabs = Kabs + (w1 * Ka[l1] + w2 * Ka[l2]) * w[q];
    Kext = Kext + (w1 * (Ka[l1] + Ks[l1]) + w2 * (Ka[l2] + Ks[l2])) * w[q];
    Ksca = Ksca + (w1 * Ks[l1] + w2 * Ks[l2]) * w[q];
  }
  const double albedo = Ksca / Kext;
  int iT = (int)(T / 1.0);
  const double wT1 = (double)(iT + 1) - T / 1.0, wT2 = T / 1.0 - (double)iT;
  if (iT < 1) iT = 1;
  if (iT > TP_TMAX - 1) iT = TP_TMAX - 1;
  const double *B1 = BB + (size_t)l1 * TP_TT, *B2 = BB + (size_t)l2 * TP_TT;
  double e = 0.0;
  for (int q = 0; q < ncomp; ++q) {
    const double *Ka = Kabs_c + (size_t)q * nlam;
    e = e + (((w1 * (wT1 * B1[iT] + wT2 * B1[iT + 1])) * Ka[l1] + (w2 * (wT1 * B2[iT] + wT2 * B2[iT + 1])) * Ka[l2]) *
             w[q]) / Kabs;
  }
  *kext = Kext;
  *emis = e * (1.0 - albedo);
}

/* start of the image ray at radius Rimg and angle phi (TraceMono.f:2243-2259) */
RT_HD void rt_ray_start(const TModel &m, double Rimg, double phi, double angle, TPkt *p) {
  const double Rout = m.R[m.nr];
  p->x = Rimg * dm_cos(phi);
  p->y = Rimg * dm_sin(phi);
  p->z = sqrt(Rout * Rout - Rimg * Rimg);
  p->edgeNr = 2;
  p->onEdge = 1;
  tp_rotate(&p->x, &p->y, &p->z, 0.0, 1.0, 0.0, angle);
  const double ct = fabs(p->z) / Rout;
  p->i = m.nr - 1;
  p->j = 1; /* a ray through the pole of the outer sphere (face-on, R = 0) keeps cell 1 */
  for (int j = 1; j <= m.nt - 1; ++j)
    if (ct < m.Theta[j - 1] && ct >= m.Theta[j]) p->j = j;
  p->vx = 0.0;
  p->vy = 0.0;
  p->vz = -1.0;
  tp_rotate(&p->vx, &p->vy, &p->vz, 0.0, 1.0, 0.0, angle);
}

/* the scattered-light field a ray pass reads: mode 2 the angular field
 * of the wavelength (f1), mode 1 the isotropic fields of the grid
 * wavelengths around it, weighted w1, w2 (TraceMono.f:255-262); albedo
 * and V per cell */
struct RtScat {
  int mode;
  SfGeom g;
  const double *thet, *f1, *f2, *albedo, *V;
  double w1, w2;
};

/* the intensity of one image ray: its path through the cells and the
 * formal solution (trace2dpath, TraceMono.f:331-474).  dens, kext, emis
 * per cell; fstar the star's flux at the wavelength; sc the scattered-light
 * field or null.  Returns the intensity; *steps the segments traced
 * (capped at maxsteps, *steps < 0 when the cap or a geometry failure ended
 * the ray). */
RT_HD double rt_ray(const TModel &m, const double *dens, const double *kext, const double *emis, double Rimg,
                    double phi, double angle, double fstar, double dimstar, int tracestar, int maxsteps, int *steps,
                    const RtScat *sc = nullptr) {
  TPkt p;
  rt_ray_start(m, Rimg, phi, angle, &p);
  const int nc = m.nt - 1;
  const bool ang = sc && sc->mode == 2;
  int irg = 1;
  if (ang) irg = sf_irg(sc->g, sc->thet, p.j, acos(fabs(p.z) / m.R[m.nr]));
  double I = 0.0, tau = 0.0, fact = 1.0;
  int hitstar = 0, n = 0;
  for (;;) {
    double v;
    int inext, jnext, irgn = irg;
    const int fail = ang ? sf_trace2edge_rg(m, sc->g, p, irg, &v, &inext, &jnext, &irgn)
                         : tp_trace2edge(m, p, &v, &inext, &jnext);
    if (fail != 0 || ++n > maxsteps) {
      *steps = -n;
      return I;
    }
    p.onEdge = 1;
    const int ip = p.i, jp = p.j;
    const double x1 = p.x, y1 = p.y;
    p.x = p.x + p.vx * v;
    p.y = p.y + p.vy * v;
    p.z = p.z + p.vz * v;
    if (ip != 0) {
      const size_t c = (size_t)ip * nc + (jp - 1);
      const double tau_e = ((v * dens[c]) * kext[c]) * RT_AU;
      double src = emis[c];
      if (sc) {
        const int side = p.z > 0.0 ? 0 : 1;
        double xs;
        if (ang) {
          xs = sf_segment_source(sc->g, sc->f1, ip, jp, irg, side, sf_jphi(x1, y1), sf_jphi(p.x, p.y),
                                 sc->albedo[c], sc->V[c]);
        } else {
          const size_t b = (c * 2 + side) * SF_NB;
          xs = ((sc->w1 * sc->f1[b] + sc->w2 * sc->f2[b]) / sc->V[c]) * sc->albedo[c];
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
      if (tau > RT_TAU_MAX) {
        *steps = n;
        return I;
      }
    }
    if (inext >= m.nr) break;
    if (inext < 0) {
      hitstar = 1;
      break;
    }
    p.i = inext;
    p.j = jnext;
    irg = irgn;
  }
  if (hitstar && tracestar) I = I + ((fstar * fact) * dimstar) / (RT_PI * ((m.R[0] * RT_AU) * (m.R[0] * RT_AU)));
  *steps = n;
  return I;
}

/* ------------------------------------------------------------ host logic */

/* tau01R for the midplane direction: the radius where the optical depth
 * from the inner edge outward along the last theta cell's mean cosine
 * reaches 0.1 (TraceMono.f:2300-2345 with trace2d's stepping,
 * MCRadiation.f:953-1105) */
static inline double rt_tau01_radius(const TModel &m, const double *dens, const double *kext) {
  const int nc = m.nt - 1;
  const double r = m.R[1], ct = (m.Theta[nc - 1] + m.Theta[nc]) / 2.0;
  TPkt p;
  p.x = sqrt(1.0 - ct * ct) * r;
  p.y = 0.0;
  p.z = ct * r;
  p.edgeNr = 1;
  p.onEdge = 1;
  p.vx = p.x / r;
  p.vy = 0.0;
  p.vz = p.z / r;
  p.i = 1;
  p.j = nc;
  const double tau0 = 0.1;
  double tau = 0.0;
  bool escape = false;
  for (int n = 0; n < 1000000; ++n) {
    double v;
    int inext, jnext;
    if (tp_trace2edge(m, p, &v, &inext, &jnext) != 0) break;
    const size_t c = (size_t)p.i * nc + (p.j - 1);
    const double tau1 = ((kext[c] * v) * dens[c]) * RT_AU;
    if (tau + tau1 > tau0) {
      v = v * (tau0 - tau) / tau1;
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
    if (inext >= m.nr || inext < 0) {
      escape = true;
      break;
    }
    p.i = inext;
    p.j = jnext;
  }
  if (escape) p.z = 0.0;
  double R01 = sqrt(p.x * p.x + p.z * p.z);
  if (R01 > m.R[m.nr - 1]) R01 = m.R[1];
  return R01;
}

/* the image radii of TracePath (TraceMono.f:2108-2222): theta_av from the
 * model's cos edges; Rfix the fixed radii (zone edges inside the grid) */
static inline std::vector<double> rt_image_radii(const TModel &m, double R01, double angle, int nj0, int nRfix,
                                                 const double *Rfix, int scat_how) {
  const int nR = m.nr, nTheta = m.nt;
  std::vector<double> ta(nTheta);
  for (int j = 1; j <= nTheta - 1; ++j) ta[j] = acos((m.Theta[j - 1] + m.Theta[j]) / 2.0);
  std::vector<double> R;
  for (int j = 1; j <= nTheta - 1; ++j) {
    R.push_back(R01 * fabs(cos(RT_PI / 2.0 - ta[j] + angle)));
    R.push_back(fabs(R01 * cos(ta[j] - RT_PI / 2.0 + angle)));
  }
  for (int j = 1; j <= nTheta - 1; ++j) {
    R.push_back(R01 * fabs(cos(RT_PI / 2.0 - ta[j])));
    R.push_back(fabs(R01 * cos(ta[j] - RT_PI / 2.0)));
  }
  if (scat_how == 2)
    for (int j = 1; j <= 180; ++j) {
      const double theta = (double)(float)j * (RT_PI / 2.0) / 181.0;
      R.push_back(m.R[1] * fabs(cos(RT_PI / 2.0 - theta)));
      for (int i = 0; i < nRfix; ++i) R.push_back(Rfix[i] * fabs(cos(RT_PI / 2.0 - theta)));
    }
  for (int i = 0; i < nRfix; ++i)
    for (int j = 1; j <= nTheta - 1; ++j) {
      R.push_back(Rfix[i] * fabs(cos(RT_PI / 2.0 - ta[j] + angle)));
      R.push_back(fabs(Rfix[i] * cos(ta[j] - RT_PI / 2.0 + angle)));
    }
  std::sort(R.begin(), R.end());
  if (nj0 > 0) {
    for (int i = 1; i <= nR - 1; ++i)
      for (int j = 1; j <= nj0; ++j)
        R.push_back(m.R[i] + (m.R[i + 1] - m.R[i]) * ((double)(float)j - 0.5) / (double)(float)nj0);
  } else {
    for (int i = 1; i <= nR - 1; i += -nj0) R.push_back(pow(10.0, log10(m.R[i] * m.R[i + 1]) / 2.0));
  }
  for (int i = 1; i <= RT_NSTAR - 1; ++i)
    R.push_back(((0.999 * m.R[0]) * (double)(float)(i - 1)) / (double)(float)(RT_NSTAR - 2));
  R.push_back(m.R[0] * (double)1.001f);
  R.push_back(m.R[nR] * (double)0.9999f);
  std::sort(R.begin(), R.end());
  /* separate equal radii (TraceMono.f:2210-2221): the scan restarts
   * from the outer end after each change, until 10 nr scans were begun */
  const int nr = (int)R.size();
  int k = 0;
  bool restart = true;
  while (restart) {
    restart = false;
    k = k + 1;
    for (int i = nr - 1; i >= 1; --i)
      if (R[i] == R[i - 1]) {
        if (i != nr - 1)
          R[i] = (R[i + 1] + R[i]) / 2.0;
        else
          R[i - 1] = (R[i - 1] + R[i]) / 2.0;
        if (k < nr * 10) {
          restart = true;
          break;
        }
      }
  }
  return R;
}

/* phi of image column k = 1..nphi (TraceMono.f:2237) */
static inline double rt_phi(int k, int nphi) {
  return 1e-5 + RT_PI * (double)((float)k - 0.5f) / (double)(float)nphi;
}

/* the trapezoid of TraceMono.f:481-493 over image[i*nphi + k] */
static inline double rt_flux(const std::vector<double> &R, int nphi, const double *image) {
  const int nr = (int)R.size();
  const double AU2 = RT_AU * RT_AU;
  double flux = 0.0;
  for (int i = 0; i < nr - 1; ++i)
    for (int k = 0; k < nphi; ++k) {
      const double w1 = (((2.0 * RT_PI) * fabs(R[i])) * AU2) / (double)(float)nphi;
      const double w2 = (((2.0 * RT_PI) * fabs(R[i + 1])) * AU2) / (double)(float)nphi;
      flux = flux + ((R[i + 1] - R[i]) * (w1 * image[(size_t)i * nphi + k] + w2 * image[(size_t)(i + 1) * nphi + k])) / 2.0;
    }
  return flux;
}

struct RtOptions {
  double angle;     /* inclination, rad */
  int nphi, nj0;    /* angles over half the image; image points per radial cell */
  int nRfix;
  const double *Rfix;
  double lam_path;  /* wavelength of the tau = 0.1 radius (0.55 micron for a spectrum) */
  int tracestar;
  double dimstar;
};

/* Backend: cells(lam0, kext[ncell], emis[ncell]) -> per-cell arrays (also
 * kept on the backend's side for the rays); field(lam0) -> the scattered
 * light field the next rays read (nothing to do without one); rays(R, phi,
 * fstar, image[nr*nphi], steps) -> the intensities.  Returns false on an
 * execution error. */
template <class Backend>
bool rt_spectrum(const TModel &m, Backend &be, const RtOptions &o, int nlam, const double *lam, const double *Fstar,
                 const double *dens, int nobs, const double *lam_obs, double *flux, std::vector<double> *Rimg,
                 std::vector<double> *image_last, int *bad_rays) {
  const int ncell = m.nr * (m.nt - 1);
  std::vector<double> kext(ncell), emis(ncell);
  if (!be.cells(o.lam_path, kext.data(), emis.data())) return false;
  const double R01 = rt_tau01_radius(m, dens, kext.data());
  *Rimg = rt_image_radii(m, R01, o.angle, o.nj0, o.nRfix, o.Rfix, m.scat_how);
  std::vector<double> phi(o.nphi);
  for (int k = 1; k <= o.nphi; ++k) phi[k - 1] = rt_phi(k, o.nphi);
  const int nr = (int)Rimg->size();
  std::vector<double> image((size_t)nr * o.nphi);
  *bad_rays = 0;
  for (int l = 0; l < nobs; ++l) {
    if (lam_obs[l] < lam[0] || lam_obs[l] > lam[nlam - 1]) { /* TraceMono.f:32-35 */
      flux[l] = 0.0;
      continue;
    }
    int l1, l2;
    double w1, w2;
    rt_lam(nlam, lam, lam_obs[l], &l1, &l2, &w1, &w2);
    const double fstar = Fstar[l1] * w1 + Fstar[l2] * w2;
    if (!be.cells(lam_obs[l], kext.data(), emis.data())) return false;
    if (!be.field(lam_obs[l])) return false;
    int bad = 0;
    if (!be.rays(*Rimg, phi, fstar, o, image.data(), &bad)) return false;
    *bad_rays += bad;
    flux[l] = rt_flux(*Rimg, o.nphi, image.data());
  }
  if (image_last) *image_last = image;
  return true;
}

/* ---- rectangular image (MakeImage, TraceMono.f:2759-3001) ----
 *
 * Sample s = (ring i, angle column j, draw k), s = (i nphi + j) nint + k,
 * places one point at a uniform position in the image cell between radii
 * R[i], R[i+1] and angles pi j/nphi, pi (j+1)/nphi, interpolates the ray
 * intensities there (bilinear in radius and angle, the angle neighbour being
 * the column on the point's side, TraceMono.f:2841-2861) and adds
 * I w2 R / (2 nint) to the pixel of the point and of its mirror image
 * -phi (TraceMono.f:2963-3001), w2 = 2 pi AU^2 (R[i+1] - R[i]) / nphi.
 *
 * The interpolation is log-linear (TraceMono.f:2931-2934, the 10**() of
 * interpolated log10 I, written here with natural logarithms) or, with
 * linear set, linear: the form the reference reaches for scattering with
 * the full Mueller matrix when the image carries no polarisation (its
 * polarised branch divides U by 2 a_l a_r = 0, number_invalid turns the
 * NaN into the linear interpolation, TraceMono.f:2862-2920).
 *
 * The two uniforms of a sample are one Philox block with key = seed and
 * counter (0, 1, s_lo, s_hi), where the reference draws ran2 in loop order.
 * key[0], key[1]: the pixel index (ix - 1) npix + (iy - 1) of the point and
 * of its mirror, npix^2 when the point falls outside the image; *val the
 * amount added to each. */
RT_HD void rt_image_sample(long long s, int nphi, int nint, const double *R, const double *image, uint64_t seed,
                           double Rmax, double pa_deg, int npix, int linear, uint32_t key[2], double *val) {
  const long long per_ring = (long long)nphi * nint;
  const int i = (int)(s / per_ring);
  const int jf = (int)((s / nint) % nphi) + 1; /* Fortran column 1..nphi */
  const uint32_t ctr[4] = {0u, 1u, (uint32_t)(unsigned long long)s, (uint32_t)((unsigned long long)s >> 32)};
  const uint32_t kk[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  px_philox4x32_10(ctr, kk, o);
  const double ranR = px_u01(o[0], o[1]), ranPhi = px_u01(o[2], o[3]);
  const double w2 = (((2.0 * RT_PI) * (RT_AU * RT_AU)) * (R[i + 1] - R[i])) / (double)(float)nphi;
  const double Rs = R[i] + (R[i + 1] - R[i]) * ranR;
  const double phi = (RT_PI * ((double)(float)(jf - 1) + ranPhi)) / (double)(float)nphi;
  int jp1, jp2 = jf;
  double wp1, wp2;
  if (ranPhi < 0.5) {
    wp1 = 0.5 - ranPhi;
    jp1 = jf - 1;
    if (jp1 == 0) jp1 = 1;
    wp2 = ranPhi + 0.5;
  } else {
    wp1 = ranPhi - 0.5;
    jp1 = jf + 1;
    if (jp1 == nphi + 1) jp1 = nphi;
    wp2 = 1.5 - ranPhi;
  }
  const double wr1 = 1.0 - ranR, wr2 = ranR;
  const double *r1 = image + (size_t)i * nphi, *r2 = image + (size_t)(i + 1) * nphi;
  const double I11 = r1[jp1 - 1], I12 = r1[jp2 - 1], I21 = r2[jp1 - 1], I22 = r2[jp2 - 1];
  double f;
  if (linear) {
    f = ((wr1 * (wp1 * I11 + wp2 * I12) + wr2 * (wp1 * I21 + wp2 * I22)) * w2) * Rs;
  } else {
    const double e = wr1 * (wp1 * dm_log(I11) + wp2 * dm_log(I12)) + wr2 * (wp1 * dm_log(I21) + wp2 * dm_log(I22));
    f = (dm_exp(e) * w2) * Rs;
  }
  *val = f / (double)(float)(2 * nint);
  const double pa = (pa_deg * RT_PI) / 180.0;
  const double npf = (double)(float)npix;
  for (int m = 0; m < 2; ++m) {
    const double a = m == 0 ? phi + pa : -phi + pa;
    const double x = (npf * (-Rs * dm_cos(a) + Rmax)) / (2.0 * Rmax) + 1.0;
    const double y = (npf * (Rs * dm_sin(a) + Rmax)) / (2.0 * Rmax) + 1.0;
    /* Fortran's ix = x truncates; ix in 1..npix  <=>  1 <= x < npix + 1 */
    if (x >= 1.0 && x < npf + 1.0 && y >= 1.0 && y < npf + 1.0)
      key[m] = (uint32_t)(((int)x - 1) * npix + ((int)y - 1));
    else
      key[m] = (uint32_t)npix * (uint32_t)npix;
  }
}

/* image radii count for the rectangular image's buffers: the size of
 * rt_image_radii's list (the model's nr, nt; nj0; nRfix; scat_how) */
static inline long long rt_image_radii_count(int nr, int nt, int nj0, int nRfix, int scat_how) {
  long long n = (nj0 > 0 ? (long long)nj0 * (nr - 1) : (long long)(nr - 2) / (-nj0) + 1);
  n += (long long)(nt - 1) * 2 * (nRfix + 2) + 1 + RT_NSTAR;
  if (scat_how == 2) n += 180LL * (nRfix + 1);
  return n;
}

#endif /* MCMAX_RT_CORE_CUH */
