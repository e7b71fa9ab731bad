/*
 * diffuse_core.cuh -- Diffuse (Diffusion.f:9-330, called after the packet
 * loop from Main.f:561-563): temperatures of optically thick cells that the
 * packets sampled poorly, from the diffusion equation for T^4 solved over
 * those cells and their neighbours.
 *
 * The same source serves the library (diffuse.cu: a backend that launches
 * kernels) and the host replay of the tests (a backend of plain loops), so
 * both run identical host logic and identical per-element arithmetic.  Every
 * a*b+c here is rounded twice (the library builds this unit with
 * --fmad=false, the replay with -ffp-contract=off).
 *
 * Layout of the linear system.  The unknowns are T^4 of a rectangular box of
 * cells (i, j) that covers every numbered cell, j fastest: row
 * r = (i - ilo) * w + (j - jlo), w = jhi - jlo + 1.  Radial neighbours are
 * rows r -+ w, theta neighbours rows r -+ 1, so the matrix is banded with
 * half-bandwidth w; box cells outside the numbered set are identity rows.
 * The reference numbers the cells in the order it meets them and calls
 * DGESV (LU with partial pivoting) on the dense N x N matrix.  Here the band
 * is eliminated without pivoting: with the stencil rows negated the matrix is
 * a nonsingular M-matrix (non-positive off-diagonals, zero row sums in the
 * stencil rows, identity rows for every kept temperature, each stencil cell
 * linked to a kept one), and every Schur complement of an M-matrix is again
 * one, so no pivot vanishes.  The two solvers agree to rounding.
 */
#ifndef MCMAX_DIFFUSE_CORE_CUH
#define MCMAX_DIFFUSE_CORE_CUH

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#ifdef __CUDACC__
#define DF_HD __host__ __device__ inline
#else
#define DF_HD static inline
#endif

#define DF_TMAX 10000
#define DF_TT (DF_TMAX + 1)
#define DF_AU ((double)1.49598e13f) /* Modules.f:8, a default-real literal */
#define DF_NITER 3                   /* Diffusion.f:24 (no flux limiter) */
#define DF_NSLOT 5                   /* stencil slots of a row, see df_fill_row */

/* KDext of cell c at temperature index iT: DiffCoeffCell (Dtable.f:97-182),
 * the Rosseland-type mean 1 / <1/(Kext - g^2 Ksca)> weighted by dB/dT,
 * trapezoids over frequency with dnu_half[l] = |nu_l - nu_l+1| / 2 */
DF_HD double df_kd_ext(int c, int iT, int nlam, int ncomp, int scattering, const double *comp_w, const double *g_c,
                       const double *Ksca_c, const double *KabsTot, const double *KscaTot, const double *dnu_half,
                       const double *BB) {
  const double *w = comp_w + (size_t)c * ncomp;
  const double *Ka = KabsTot + (size_t)c * nlam, *Ks = KscaTot + (size_t)c * nlam;
  double int1 = 0.0, int2 = 0.0, e0 = 0.0, b0 = 0.0;
  for (int l = 0; l < nlam; ++l) {
    double g = 0.0;
    for (int q = 0; q < ncomp; ++q) g = g + (g_c[(size_t)q * nlam + l] * Ksca_c[(size_t)q * nlam + l]) * w[q];
    g = g / Ks[l];
    if (!scattering) g = 0.0;
    const double Kext = Ka[l] + Ks[l];
    const double b1 = BB[(size_t)l * DF_TT + iT + 1] - BB[(size_t)l * DF_TT + iT];
    const double e1 = b1 / (Kext - (g * g) * Ks[l]);
    if (l > 0) {
      int1 = int1 + dnu_half[l - 1] * (e0 + e1);
      int2 = int2 + dnu_half[l - 1] * (b0 + b1);
    }
    e0 = e1;
    b0 = b1;
  }
  return int2 / int1;
}

/* ---- banded elimination, one element per call ----
 * band[r*(2w+1) + (c - r + w)] holds A(r, c); b is the right-hand side.
 * Step k: the multipliers of rows k+1..k+m (m = min(w, nb-1-k)) ... */
DF_HD double df_elim_mult(const double *band, int w, int k, int t) {
  const size_t W = 2 * (size_t)w + 1;
  return band[(size_t)(k + 1 + t) * W + (size_t)(w - 1 - t)] / band[(size_t)k * W + w];
}

/* ... then element e of the (m) x (m+1) update: row k+1+e/(m+1), column
 * k+1+e%(m+1), the last column being the right-hand side */
DF_HD void df_elim_update(double *band, double *b, int w, int k, int m, int e, const double *lm) {
  const size_t W = 2 * (size_t)w + 1;
  const int a = e / (m + 1), col = e - a * (m + 1);
  const double l = lm[a];
  if (l == 0.0) return;
  const int r = k + 1 + a;
  if (col < m) {
    const int c = k + 1 + col;
    double *x = band + (size_t)r * W + (size_t)(c - r + w);
    *x = *x - l * band[(size_t)k * W + (size_t)(c - k + w)];
  } else {
    b[r] = b[r] - l * b[k];
  }
}

/* back substitution, step k (descending): x_k = b_k / A(k,k), then each row
 * r in [k-w, k) drops A(r,k) x_k */
DF_HD double df_back_x(const double *band, const double *b, int w, int k) {
  return b[k] / band[(size_t)k * (2 * (size_t)w + 1) + w];
}
DF_HD void df_back_update(const double *band, double *b, int w, int k, int r, double xk) {
  b[r] = b[r] - band[(size_t)r * (2 * (size_t)w + 1) + (size_t)(k - r + w)] * xk;
}

/* scatter the stencil slots of row r into the zeroed band: centre, inner
 * and outer radial neighbour (r -+ w), polar and midplane-side theta
 * neighbour (r -+ 1) */
DF_HD void df_fill_row(double *band, int w, int r, const double *coef) {
  const size_t W = 2 * (size_t)w + 1, o = (size_t)r * W;
  const int off[DF_NSLOT] = {w, 0, 2 * w, w - 1, w + 1};
  for (int s = 0; s < DF_NSLOT; ++s)
    if (coef[s] != 0.0) band[o + (size_t)off[s]] = coef[s];
}

/* ------------------------------------------------------------ host logic */

struct DfGrid {
  int nr, nt;             /* D%nR (edges R[0..nr]) and D%nTheta */
  const double *R;        /* nr+1, AU */
  const double *Theta;    /* nt, cos theta edges, Theta[0] = 1 */
  const double *dens;     /* ncell */
  int ncomp;
  const double *comp_w;   /* ncell*ncomp */
};

struct DfStats {
  int ncor = 0;           /* cells selected for diffusion (Diffusion.f:45-49) */
  int nunknown = 0;       /* numbered cells */
  int nsolved = 0;        /* cells given a diffusion temperature in the last pass */
  int nb = 0, w = 0;      /* box rows and half-bandwidth */
  int failed = 0;         /* passes whose elimination met a zero or non-finite pivot */
};

/* Backend: kd(n, cells, iTs, out) -> KDext; kp(n, cells, iTs, out) ->
 * Planck mean of the cell's mixture; solve(nb, w, coef[nb*5], rhs[nb],
 * x[nb]) -> 0, or a nonzero code after a zero/non-finite pivot.  Each returns
 * false on an execution error. */
template <class Backend>
bool df_diffuse(const DfGrid &g, Backend &be, int nphotmin, double dtmax, double factRW, const int32_t *Ni,
                const double *dT, double *T, double *EJv, DfStats *st) {
  const int nR = g.nr, nTheta = g.nt, nc = nTheta - 1, ncell = nR * nc;
  auto C = [nc](int i, int j) { return i * nc + (j - 1); };   /* reference (i, j), j = 1..nTheta-1 */
  *st = DfStats();
  if (nR < 4 || nTheta < 3) return true;

  /* thick flags as InitRandomWalk sets them (RandomWalk.f:172-190) */
  std::vector<unsigned char> thick(ncell, 0);
  {
    std::vector<int> cells, iTs;
    for (int c = nc; c < ncell; ++c)
      for (int iT = 100; iT <= 1600; iT += 500) {
        cells.push_back(c);
        iTs.push_back(iT);
      }
    std::vector<double> kd(cells.size());
    if (!cells.empty() && !be.kd((int)cells.size(), cells.data(), iTs.data(), kd.data())) return false;
    for (size_t k = 0; k < cells.size(); ++k) {
      const int c = cells[k], i = c / nc;
      const double lr = 1.0 / ((DF_AU * kd[k]) * g.dens[c]);
      if ((g.R[i + 1] - g.R[i]) > factRW * lr) thick[c] = 1;
    }
  }

  /* cells to diffuse and their neighbours (Diffusion.f:39-76) */
  std::vector<unsigned char> assigned(ncell, 0);
  for (int i = 2; i <= nR - 2; ++i)
    for (int j = 2; j <= nTheta - 1; ++j) {
      const int c = C(i, j);
      if (!(Ni[c] < nphotmin || (dT[c] / T[c]) > dtmax)) continue;
      if (!(thick[c] || Ni[c] <= 1)) continue;
      st->ncor++;
      assigned[c] = assigned[C(i - 1, j)] = assigned[C(i + 1, j)] = assigned[C(i, j - 1)] = 1;
      if (j != nTheta - 1) assigned[C(i, j + 1)] = 1;
    }
  int ilo = nR, ihi = -1, jlo = nTheta, jhi = -1;
  std::vector<int> num;   /* numbered cells, box order */
  for (int i = 1; i <= nR - 1; ++i)
    for (int j = 1; j <= nTheta - 1; ++j)
      if (assigned[C(i, j)]) {
        num.push_back(C(i, j));
        ilo = std::min(ilo, i); ihi = std::max(ihi, i);
        jlo = std::min(jlo, j); jhi = std::max(jhi, j);
      }
  st->nunknown = (int)num.size();
  if (num.empty()) return true;
  const int w = jhi - jlo + 1, nb = (ihi - ilo + 1) * w;
  st->nb = nb;
  st->w = w;
  auto row = [&](int i, int j) { return (i - ilo) * w + (j - jlo); };

  /* cell centres: D%R_av in cm (Init.f:2873), D%theta_av (Init.f:2889) */
  std::vector<double> r_av(nR), t_av(nTheta);
  for (int i = 1; i <= nR - 1; ++i) r_av[i] = DF_AU * pow(10.0, (log10(g.R[i]) + log10(g.R[i + 1])) / 2.0);
  for (int j = 1; j <= nTheta - 1; ++j) t_av[j] = acos((g.Theta[j - 1] + g.Theta[j]) / 2.0);
  const double pi = 3.14159265358979323846;

  const int n = (int)num.size();
  std::vector<int> iTs(n);
  std::vector<double> kd(n), Dc(ncell, 0.0), coef((size_t)nb * DF_NSLOT), rhs(nb), x(nb);
  std::vector<unsigned char> ok(ncell, 1);
  for (int it = 0; it < DF_NITER; ++it) {
    /* Rosseland diffusion coefficient per numbered cell (Diffusion.f:124-151) */
    for (int k = 0; k < n; ++k) {
      int iT = (int)(T[num[k]] / 1.0);
      if (iT <= 1) iT = 1;
      if (iT >= DF_TMAX - 1) iT = DF_TMAX - 1;
      iTs[k] = iT;
    }
    if (!be.kd(n, num.data(), iTs.data(), kd.data())) return false;
    for (int k = 0; k < n; ++k) {
      const int c = num[k], i = c / nc, j = c % nc + 1;
      double dens = 0.0;
      for (int q = 0; q < g.ncomp; ++q) dens = dens + g.comp_w[(size_t)c * g.ncomp + q] * g.dens[c];
      Dc[c] = 1.0 / (kd[k] * dens);
      if (((g.R[nR] - g.R[i]) * DF_AU / Dc[c]) < 2.0) thick[c] = 0;
      if (Ni[c] < nphotmin || (dT[c] / T[c]) > dtmax) {
        ok[c] = 0;
        if (i == 1 || i == nR - 1 || j == 1) ok[c] = 1;
        if (!thick[c] && Ni[c] > 1) ok[c] = 1;
      } else {
        ok[c] = 1;
      }
    }
    /* A cell that turns unresolved only in a later pass (its dT/T grew with
     * the new T) may have neighbours outside the numbered set; the reference
     * then reads unset entries (number = 0).  Such a cell keeps its
     * temperature here. */
    for (int k = 0; k < n; ++k) {
      const int c = num[k], i = c / nc, j = c % nc + 1;
      if (ok[c]) continue;
      if (!assigned[C(i - 1, j)] || !assigned[C(i + 1, j)] || !assigned[C(i, j - 1)] ||
          (j != nTheta - 1 && !assigned[C(i, j + 1)]))
        ok[c] = 1;
    }
    /* rows of the system (Diffusion.f:197-256) */
    std::fill(coef.begin(), coef.end(), 0.0);
    std::fill(rhs.begin(), rhs.end(), 0.0);
    for (int r = 0; r < nb; ++r) coef[(size_t)r * DF_NSLOT] = 1.0;
    st->nsolved = 0;
    for (int k = 0; k < n; ++k) {
      const int c = num[k], i = c / nc, j = c % nc + 1, r = row(i, j);
      double *q = &coef[(size_t)r * DF_NSLOT];
      if (ok[c]) {
        rhs[r] = (T[c] * T[c]) * (T[c] * T[c]);
        continue;
      }
      st->nsolved++;
      q[0] = 0.0;
      /* radial part */
      const double r0 = r_av[i], rm = r_av[i - 1], rp = r_av[i + 1];
      double dx0 = log(rp / rm), dx1 = log(rp / r0), dx2 = log(r0 / rm);
      double f1 = Dc[C(i + 1, j)] * rp, f2 = Dc[C(i - 1, j)] * rm;
      const double r03 = (r0 * r0) * r0;
      q[1] = q[1] + f2 / ((dx2 * dx0) * r03);
      q[0] = q[0] - f2 / ((dx2 * dx0) * r03);
      q[2] = q[2] + f1 / ((dx1 * dx0) * r03);
      q[0] = q[0] - f1 / ((dx1 * dx0) * r03);
      /* theta part; at the midplane the cell is its own mirror neighbour */
      const bool mid = (j == nTheta - 1);
      const double t0 = t_av[j], tjm = mid ? pi - t_av[j] : t_av[j + 1], tjp = t_av[j - 1];
      dx0 = tjp - tjm;
      dx1 = tjp - t0;
      dx2 = t0 - tjm;
      f1 = Dc[C(i, j - 1)] * sin(tjp);
      f2 = Dc[mid ? c : C(i, j + 1)] * sin(tjm);
      const double r02 = r0 * r0, st0 = sin(t0);
      double *qm = mid ? &q[0] : &q[4];
      *qm = *qm + f2 / (((dx2 * dx0) * r02) * st0);
      q[0] = q[0] - f2 / (((dx2 * dx0) * r02) * st0);
      q[3] = q[3] + f1 / (((dx1 * dx0) * r02) * st0);
      q[0] = q[0] - f1 / (((dx1 * dx0) * r02) * st0);
    }
    int code = 0;
    if (!be.solve(nb, w, coef.data(), rhs.data(), x.data(), &code)) return false;
    if (code != 0) {
      /* DGESV's INFO > 0: the right-hand side stays unsolved, zero in every
       * stencil row, so those temperatures stay as they are */
      st->failed++;
      std::copy(rhs.begin(), rhs.end(), x.begin());
    }
    /* new temperatures and emission of the solved cells (Diffusion.f:265-288) */
    std::vector<int> upd, updT;
    for (int k = 0; k < n; ++k) {
      const int c = num[k], i = c / nc, j = c % nc + 1;
      if (ok[c]) continue;
      const double T4 = x[row(i, j)];
      if (T4 > 0.0) T[c] = pow(T4, 0.25);
      if (T4 < 0.0) T[c] = 1.0;
      int iT = (int)(T[c] / 1.0);
      if (iT <= 1) iT = 1;
      if (iT >= DF_TMAX - 1) iT = DF_TMAX - 1;
      upd.push_back(c);
      updT.push_back(iT);
      if (T[c] > (double)(DF_TMAX - 1)) T[c] = (double)(DF_TMAX - 1);
      if (T[c] < 1.0) T[c] = 1.0;
      if (!(T[c] == T[c]) || isinf(T[c])) T[c] = 1.0;
    }
    if (EJv && !upd.empty()) {
      std::vector<double> e(upd.size());
      if (!be.kp((int)upd.size(), upd.data(), updT.data(), e.data())) return false;
      for (size_t k = 0; k < upd.size(); ++k) EJv[upd[k]] = e[k];
    }
  }
  return true;
}

/* the band solve as serial loops over the same per-element functions the
 * kernel runs (host backend and replay) */
static inline int df_band_solve_host(int nb, int w, const double *coef, const double *rhs, double *x) {
  const size_t W = 2 * (size_t)w + 1;
  std::vector<double> band((size_t)nb * W, 0.0), b(rhs, rhs + nb), lm(w > 0 ? w : 1);
  for (int r = 0; r < nb; ++r) df_fill_row(band.data(), w, r, coef + (size_t)r * DF_NSLOT);
  int code = 0;
  for (int k = 0; k < nb; ++k) {
    const double piv = band[(size_t)k * W + w];
    if (code == 0 && (!(fabs(piv) > 0.0) || isinf(piv))) code = k + 1;
    const int m = std::min(w, nb - 1 - k);
    if (m <= 0) break;
    for (int t = 0; t < m; ++t) lm[t] = df_elim_mult(band.data(), w, k, t);
    for (int e = 0; e < m * (m + 1); ++e) df_elim_update(band.data(), b.data(), w, k, m, e, lm.data());
  }
  for (int k = nb - 1; k >= 0; --k) {
    const double xk = df_back_x(band.data(), b.data(), w, k);
    for (int r = std::max(0, k - w); r < k; ++r) df_back_update(band.data(), b.data(), w, k, r, xk);
    x[k] = xk;
  }
  return code;
}

#endif /* MCMAX_DIFFUSE_CORE_CUH */
