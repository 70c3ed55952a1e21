// Small dense solves shared by the solve kernels.
#pragma once

namespace flpr {

constexpr int kMaxNt = 10;

// z = A^-1 e1 for symmetric A (nt x nt, row-major), LDL' without pivoting;
// falls back to Gaussian elimination with partial pivoting when a pivot is
// zero or not finite.  Returns false if A is singular.
__device__ __forceinline__ bool solve_e1(int nt, double A[kMaxNt][kMaxNt], double z[kMaxNt]) {
  double Lm[kMaxNt][kMaxNt];
  double D[kMaxNt];
  bool ok = true;
  for (int j = 0; j < nt && ok; ++j) {
    double dj = A[j][j];
    for (int k = 0; k < j; ++k) dj -= Lm[j][k] * Lm[j][k] * D[k];
    if (!(fabs(dj) > 0.0) || !isfinite(dj)) {
      ok = false;
      break;
    }
    D[j] = dj;
    Lm[j][j] = 1.0;
    for (int i = j + 1; i < nt; ++i) {
      double v = A[i][j];
      for (int k = 0; k < j; ++k) v -= Lm[i][k] * Lm[j][k] * D[k];
      Lm[i][j] = v / dj;
    }
  }
  if (ok) {
    // L y = e1 ; D w = y ; L' z = w
    double y[kMaxNt];
    for (int i = 0; i < nt; ++i) {
      double v = (i == 0) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) v -= Lm[i][k] * y[k];
      y[i] = v;
    }
    for (int i = 0; i < nt; ++i) y[i] /= D[i];
    for (int i = nt - 1; i >= 0; --i) {
      double v = y[i];
      for (int k = i + 1; k < nt; ++k) v -= Lm[k][i] * z[k];
      z[i] = v;
    }
    return true;
  }
  // Gaussian elimination with partial pivoting on [A | e1]
  double B[kMaxNt][kMaxNt + 1];
  for (int i = 0; i < nt; ++i) {
    for (int j = 0; j < nt; ++j) B[i][j] = A[i][j];
    B[i][nt] = (i == 0) ? 1.0 : 0.0;
  }
  for (int c = 0; c < nt; ++c) {
    int piv = c;
    for (int r = c + 1; r < nt; ++r)
      if (fabs(B[r][c]) > fabs(B[piv][c])) piv = r;
    if (!(fabs(B[piv][c]) > 0.0)) return false;
    if (piv != c)
      for (int j = 0; j <= nt; ++j) {
        double t = B[c][j];
        B[c][j] = B[piv][j];
        B[piv][j] = t;
      }
    for (int r = c + 1; r < nt; ++r) {
      double f = B[r][c] / B[c][c];
      for (int j = c; j <= nt; ++j) B[r][j] -= f * B[c][j];
    }
  }
  for (int i = nt - 1; i >= 0; --i) {
    double v = B[i][nt];
    for (int k = i + 1; k < nt; ++k) v -= B[i][k] * z[k];
    z[i] = v / B[i][i];
  }
  return true;
}


// z = (S + lam I)^-1 e1 with S given packed lower-triangular column-major.
__device__ __forceinline__ bool solve_e1_packed(int nt, const double* Ap, double lam, double* z) {
  double A[kMaxNt][kMaxNt];
  int k = 0;
  for (int j = 0; j < nt; ++j)
    for (int i = j; i < nt; ++i) {
      A[i][j] = Ap[k];
      A[j][i] = Ap[k];
      ++k;
    }
  for (int i = 0; i < nt; ++i) A[i][i] += lam;
  double zz[kMaxNt];
  bool ok = solve_e1(nt, A, zz);
  for (int i = 0; i < nt; ++i) z[i] = zz[i];
  return ok;
}

}  // namespace flpr
