/*
 * oracle_diffuse.c -- CPU restatement of Diffuse (Diffusion.f:9-330), test
 * infrastructure only: the checker of mcg_diffuse, never linked by the
 * product.
 *
 * It follows the reference's own order: cells numbered as the selection
 * loop meets them (Diffusion.f:39-76), the dense N x N matrix of
 * Diffusion.f:197-256, and DGESV (Lapack.f:6429) restated as LU with
 * partial pivoting (the column scan of IDAMAX takes the first largest
 * |a|, row interchange, the column scaled by the reciprocal pivot, rank-one
 * update: DGETF2, Lapack.f:6541) followed by the row interchanges and the
 * two triangular solves of DGETRS.  The reference's DGETRF runs the same
 * elimination in blocks of ILAENV's size; the blocking changes rounding
 * only.  No flux limiter (FLD), no QHP grains, thermal contact.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define AU_D ((double)1.49598e13f) /* Modules.f:8 */

/* DGESV: A (n x n, row-major) and b overwritten; returns INFO (0, or the
 * 1-based column of the first exactly zero pivot; b is then unsolved) */
static int dgesv(int n, double *A, double *b) {
  int *piv = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int info = 0;
  for (int j = 0; j < n; ++j) {
    int p = j;
    double amax = fabs(A[(size_t)j * n + j]);
    for (int i = j + 1; i < n; ++i)
      if (fabs(A[(size_t)i * n + j]) > amax) {
        amax = fabs(A[(size_t)i * n + j]);
        p = i;
      }
    piv[j] = p;
    if (A[(size_t)p * n + j] != 0.0) {
      if (p != j)
        for (int k = 0; k < n; ++k) {
          double t = A[(size_t)j * n + k];
          A[(size_t)j * n + k] = A[(size_t)p * n + k];
          A[(size_t)p * n + k] = t;
        }
      const double ajj = A[(size_t)j * n + j];
      if (fabs(ajj) >= 2.2250738585072014e-308) {
        const double rcp = 1.0 / ajj;
        for (int i = j + 1; i < n; ++i) A[(size_t)i * n + j] *= rcp;
      } else {
        for (int i = j + 1; i < n; ++i) A[(size_t)i * n + j] /= ajj;
      }
    } else if (info == 0) {
      info = j + 1;
    }
    for (int k = j + 1; k < n; ++k) {
      const double t = -A[(size_t)j * n + k];
      if (t == 0.0) continue;
      for (int i = j + 1; i < n; ++i) A[(size_t)i * n + k] = A[(size_t)i * n + k] + A[(size_t)i * n + j] * t;
    }
  }
  if (info == 0) {
    for (int j = 0; j < n; ++j)
      if (piv[j] != j) {
        double t = b[j];
        b[j] = b[piv[j]];
        b[piv[j]] = t;
      }
    for (int j = 0; j < n; ++j)
      if (b[j] != 0.0)
        for (int i = j + 1; i < n; ++i) b[i] = b[i] - b[j] * A[(size_t)i * n + j];
    for (int j = n - 1; j >= 0; --j)
      if (b[j] != 0.0) {
        b[j] = b[j] / A[(size_t)j * n + j];
        for (int i = 0; i < j; ++i) b[i] = b[i] - b[j] * A[(size_t)i * n + j];
      }
  }
  free(piv);
  return info;
}

int orc_diffuse(int nr, int nt, const double *R, const double *Theta, const double *dens, int ncomp,
                const double *comp_w, const double *KDext, const double *KpCell, int kp_uniform, uint8_t *thick,
                int nphotmin, double dtmax, const int32_t *Ni, const double *dT, double *T, double *EJv,
                int *stats) {
  const int nR = nr, nTheta = nt, nc = nt - 1, TT = ORC_TMAX + 1;
  const double pi = 3.14159265358979323846;
#define CI(i, j) ((i) * nc + ((j) - 1))
  stats[0] = stats[1] = stats[2] = stats[3] = 0;
  int *number = (int *)calloc((size_t)nR * nc, sizeof(int));
  int N = 0, ncor = 0;
  for (int i = 2; i <= nR - 2; ++i)
    for (int j = 2; j <= nTheta - 1; ++j) {
      const int c = CI(i, j);
      if (!(Ni[c] < nphotmin || (dT[c] / T[c]) > dtmax)) continue;
      if (!(thick[c] || Ni[c] <= 1)) continue;
      ncor++;
      const int nb[5][2] = {{i, j}, {i - 1, j}, {i + 1, j}, {i, j - 1}, {i, j + 1}};
      for (int q = 0; q < 5; ++q) {
        if (q == 4 && j == nTheta - 1) continue;
        const int cc = CI(nb[q][0], nb[q][1]);
        if (!number[cc]) number[cc] = ++N;
      }
    }
  stats[0] = ncor;
  stats[1] = N;
  if (N < 1) {
    free(number);
    return 0;
  }
  int *celi = (int *)malloc(sizeof(int) * (N + 1)), *celj = (int *)malloc(sizeof(int) * (N + 1));
  double *r = (double *)malloc(sizeof(double) * (N + 1)), *t = (double *)malloc(sizeof(double) * (N + 1));
  double *Dc = (double *)malloc(sizeof(double) * (N + 1)), *T4 = (double *)malloc(sizeof(double) * (N + 1));
  uint8_t *ok = (uint8_t *)malloc((size_t)N + 1);
  double *M = (double *)malloc(sizeof(double) * (size_t)N * N);
  for (int i = 1; i <= nR - 1; ++i)
    for (int j = 1; j <= nTheta - 1; ++j) {
      const int k = number[CI(i, j)];
      if (!k) continue;
      celi[k] = i;
      celj[k] = j;
      r[k] = AU_D * pow(10.0, (log10(R[i]) + log10(R[i + 1])) / 2.0);   /* Init.f:2873 */
      t[k] = acos((Theta[j - 1] + Theta[j]) / 2.0);                     /* Init.f:2889 */
    }
  for (int iter = 0; iter < 3; ++iter) {
    for (int k = 1; k <= N; ++k) {
      const int c = CI(celi[k], celj[k]);
      int iT = (int)(T[c] / 1.0);
      if (iT <= 1) iT = 1;
      if (iT >= ORC_TMAX - 1) iT = ORC_TMAX - 1;
      const double Kext = KDext[(size_t)c * TT + iT] - 0.0;
      double d = 0.0;
      for (int q = 0; q < ncomp; ++q) d = d + comp_w[(size_t)c * ncomp + q] * dens[c];
      Dc[k] = 1.0 / (Kext * d);
      if (((R[nR] - R[celi[k]]) * AU_D / Dc[k]) < 2.0) thick[c] = 0;
      if (Ni[c] < nphotmin || (dT[c] / T[c]) > dtmax) {
        ok[k] = 0;
        if (celi[k] == 1 || celi[k] == nR - 1 || celj[k] == 1) ok[k] = 1;
        if (!thick[c] && Ni[c] > 1) ok[k] = 1;
      } else {
        ok[k] = 1;
      }
    }
    /* a cell unresolved only in a later pass whose neighbours are not all
     * numbered keeps its temperature (the reference reads unset entries) */
    for (int k = 1; k <= N; ++k) {
      const int i = celi[k], j = celj[k];
      if (!ok[k] && (!number[CI(i - 1, j)] || !number[CI(i + 1, j)] || !number[CI(i, j - 1)] ||
                     (j != nTheta - 1 && !number[CI(i, j + 1)])))
        ok[k] = 1;
    }
    memset(M, 0, sizeof(double) * (size_t)N * N);
    int nsolved = 0;
    for (int k = 1; k <= N; ++k) {
      double *row = M + (size_t)(k - 1) * N;
      const int c = CI(celi[k], celj[k]);
      if (ok[k]) {
        row[k - 1] = 1.0;
        T4[k] = (T[c] * T[c]) * (T[c] * T[c]);
        continue;
      }
      nsolved++;
      const int i = celi[k], j = celj[k];
      int j0 = number[CI(i, j)], jm = number[CI(i - 1, j)], jp = number[CI(i + 1, j)];
      double dx0 = log(r[jp] / r[jm]), dx1 = log(r[jp] / r[j0]), dx2 = log(r[j0] / r[jm]);
      double f1 = Dc[jp] * r[jp], f2 = Dc[jm] * r[jm];
      const double r3 = (r[j0] * r[j0]) * r[j0];
      row[jm - 1] = row[jm - 1] + f2 / ((dx2 * dx0) * r3);
      row[j0 - 1] = row[j0 - 1] - f2 / ((dx2 * dx0) * r3);
      row[jp - 1] = row[jp - 1] + f1 / ((dx1 * dx0) * r3);
      row[j0 - 1] = row[j0 - 1] - f1 / ((dx1 * dx0) * r3);
      double tjm;
      if (j != nTheta - 1) {
        jm = number[CI(i, j + 1)];
        tjm = t[jm];
      } else {
        jm = j0;
        tjm = pi - t[jm];
      }
      jp = number[CI(i, j - 1)];
      dx0 = t[jp] - tjm;
      dx1 = t[jp] - t[j0];
      dx2 = t[j0] - tjm;
      f1 = Dc[jp] * sin(t[jp]);
      f2 = Dc[jm] * sin(tjm);
      const double r2 = r[j0] * r[j0], s0 = sin(t[j0]);
      row[jm - 1] = row[jm - 1] + f2 / (((dx2 * dx0) * r2) * s0);
      row[j0 - 1] = row[j0 - 1] - f2 / (((dx2 * dx0) * r2) * s0);
      row[jp - 1] = row[jp - 1] + f1 / (((dx1 * dx0) * r2) * s0);
      row[j0 - 1] = row[j0 - 1] - f1 / (((dx1 * dx0) * r2) * s0);
      T4[k] = 0.0;
    }
    stats[2] = nsolved;
    if (dgesv(N, M, T4 + 1) != 0) stats[3]++;
    for (int k = 1; k <= N; ++k) {
      if (ok[k]) continue;
      const int c = CI(celi[k], celj[k]);
      if (T4[k] > 0.0) T[c] = pow(T4[k], 0.25);
      if (T4[k] < 0.0) T[c] = 1.0;
      int iT = (int)(T[c] / 1.0);
      if (iT <= 1) iT = 1;
      if (iT >= ORC_TMAX - 1) iT = ORC_TMAX - 1;
      if (EJv) EJv[c] = KpCell[(kp_uniform ? (size_t)0 : (size_t)c * TT) + iT];
      if (T[c] > (double)(ORC_TMAX - 1)) T[c] = (double)(ORC_TMAX - 1);
      if (T[c] < 1.0) T[c] = 1.0;
      if (isnan(T[c]) || isinf(T[c])) T[c] = 1.0;
    }
  }
#undef CI
  free(number); free(celi); free(celj); free(r); free(t); free(Dc); free(T4); free(ok); free(M);
  return 0;
}
