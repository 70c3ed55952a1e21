// Small dense solves shared by the solve kernels.
#pragma once

namespace flpr {

constexpr int kMaxNt = 10;

}  // namespace flpr

namespace flpr {

// Compile-time sized variant (registers only): z = (S + lam I)^-1 e1, S packed
// lower-triangular column-major.  LDL' without pivoting; Gaussian elimination
// with partial pivoting when a pivot vanishes.  Returns false if singular.
template <int NT>
__device__ __forceinline__ bool solve_e1_fixed(const double* Ap, double lam, double (&z)[NT]) {
  double A[NT][NT];
  {
    int k = 0;
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int i = j; i < NT; ++i) {
        A[i][j] = Ap[k];
        A[j][i] = Ap[k];
        ++k;
      }
  }
#pragma unroll
  for (int i = 0; i < NT; ++i) A[i][i] += lam;
  double Lm[NT][NT];
  double D[NT];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    double dj = A[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) dj -= Lm[j][k] * Lm[j][k] * D[k];
    ok = ok && (fabs(dj) > 0.0) && isfinite(dj);
    D[j] = dj;
#pragma unroll
    for (int i = j + 1; i < NT; ++i) {
      double v = A[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= Lm[i][k] * Lm[j][k] * D[k];
      Lm[i][j] = v / dj;
    }
  }
  if (ok) {
    double y[NT];
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      double v = (i == 0) ? 1.0 : 0.0;
#pragma unroll
      for (int k = 0; k < i; ++k) v -= Lm[i][k] * y[k];
      y[i] = v;
    }
#pragma unroll
    for (int i = 0; i < NT; ++i) y[i] /= D[i];
#pragma unroll
    for (int i = NT - 1; i >= 0; --i) {
      double v = y[i];
#pragma unroll
      for (int k = i + 1; k < NT; ++k) v -= Lm[k][i] * z[k];
      z[i] = v;
    }
    return true;
  }
  // Gaussian elimination with partial pivoting on [A | e1]; row swaps are
  // done with selects so every index stays compile-time
  double B[NT][NT + 1];
#pragma unroll
  for (int i = 0; i < NT; ++i) {
#pragma unroll
    for (int j = 0; j < NT; ++j) B[i][j] = A[i][j];
    B[i][NT] = (i == 0) ? 1.0 : 0.0;
  }
  bool singular = false;
#pragma unroll
  for (int c = 0; c < NT; ++c) {
    double best = fabs(B[c][c]);
    int piv = c;
#pragma unroll
    for (int r = c + 1; r < NT; ++r)
      if (fabs(B[r][c]) > best) {
        best = fabs(B[r][c]);
        piv = r;
      }
    singular = singular || !(best > 0.0);
#pragma unroll
    for (int r = c + 1; r < NT; ++r) {
      if (r == piv) {
#pragma unroll
        for (int j = 0; j <= NT; ++j) {
          const double t = B[c][j];
          B[c][j] = B[r][j];
          B[r][j] = t;
        }
      }
    }
#pragma unroll
    for (int r = c + 1; r < NT; ++r) {
      const double f = B[r][c] / B[c][c];
#pragma unroll
      for (int j = c; j <= NT; ++j) B[r][j] -= f * B[c][j];
    }
  }
#pragma unroll
  for (int i = NT - 1; i >= 0; --i) {
    double v = B[i][NT];
#pragma unroll
    for (int k = i + 1; k < NT; ++k) v -= B[i][k] * z[k];
    z[i] = v / B[i][i];
  }
  return !singular;
}

}  // namespace flpr
