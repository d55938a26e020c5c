// u3b_kabsch.cc -- stand-in for the Fortran u3b_ (gpudocksm-rem-1.2/src/rmsd.f)
// that the reference's ligand loader calls to drop near-duplicate conformers
// (load.C:342-417).  gfortran is not available, so the weighted least-squares
// superposition residual is computed here from Kabsch (1976) via Horn's
// quaternion form (1987): E = sum w(|x|^2 + |y|^2) - 2 lambda_max(N), with
// both sets centred.  Only rms is produced (the loader uses nothing else);
// u and t are set to the identity and the centroid difference.
#include <cmath>

#include "size.h"

static void jacobi4(double a[4][4], double *lmax) {
  double v[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0;
    for (int i = 0; i < 4; ++i)
      for (int j = i + 1; j < 4; ++j) off += a[i][j] * a[i][j];
    if (off < 1e-22) break;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) {
        if (std::fabs(a[p][q]) < 1e-30) continue;
        const double th = (a[q][q] - a[p][p]) / (2 * a[p][q]);
        const double t = (th >= 0 ? 1 : -1) / (std::fabs(th) + std::sqrt(th * th + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 4; ++k) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 4; ++k) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 4; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  double m = a[0][0];
  for (int i = 1; i < 4; ++i) m = a[i][i] > m ? a[i][i] : m;
  *lmax = m;
}

extern "C" void u3b_(float (*w)[MAXLIG], float (*x)[MAXLIG][3], float (*y)[MAXLIG][3], int *n,
                     int *mode, float *rms, float (*u)[3][3], float (*t)[3], int *ier) {
  (void)mode;
  const int N = *n;
  double cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0}, ws = 0;
  for (int i = 0; i < N; ++i) {
    ws += (*w)[i];
    for (int k = 0; k < 3; ++k) {
      cx[k] += (*w)[i] * (*x)[i][k];
      cy[k] += (*w)[i] * (*y)[i][k];
    }
  }
  for (int k = 0; k < 3; ++k) {
    cx[k] /= ws;
    cy[k] /= ws;
  }
  double S[3][3] = {{0}}, e0 = 0;
  for (int i = 0; i < N; ++i) {
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      a[k] = (*x)[i][k] - cx[k];
      b[k] = (*y)[i][k] - cy[k];
      e0 += (*w)[i] * (a[k] * a[k] + b[k] * b[k]);
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) S[r][c] += (*w)[i] * a[r] * b[c];
  }
  double Nm[4][4] = {
      {S[0][0] + S[1][1] + S[2][2], S[1][2] - S[2][1], S[2][0] - S[0][2], S[0][1] - S[1][0]},
      {S[1][2] - S[2][1], S[0][0] - S[1][1] - S[2][2], S[0][1] + S[1][0], S[2][0] + S[0][2]},
      {S[2][0] - S[0][2], S[0][1] + S[1][0], -S[0][0] + S[1][1] - S[2][2], S[1][2] + S[2][1]},
      {S[0][1] - S[1][0], S[2][0] + S[0][2], S[1][2] + S[2][1], -S[0][0] - S[1][1] + S[2][2]}};
  double lmax = 0;
  jacobi4(Nm, &lmax);
  double e = e0 - 2 * lmax;
  *rms = (float)(e < 0 ? 0 : e);
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) (*u)[r][c] = r == c ? 1.f : 0.f;
    (*t)[r] = (float)(cy[r] - cx[r]);
  }
  *ier = 0;
}
