/*
 * C restatement of the reference's CPU hot loops -- TEST INFRASTRUCTURE ONLY
 * (checker and CPU baseline; never part of the fastlpr_b200 product).
 *
 * oracle_spread: Gaussian gridding of fused_spreading_{1,2,3}d_real
 *   (fastLPR_py/src/fastlpr/spreading_fused.py:48-129): for every point in
 *   input order, m = round-half-even(xmod/hx) per axis, taps j in
 *   [-msp, msp], weight exp(-sum_d diff_d^2/(4 tau_d)) with
 *   diff_d = xmod_d - hx_d*(m_d+j_d), index (m+j) mod L, row-major.
 *   Serial accumulation in float64, like the reference.
 * oracle_interp: clamped multilinear interpolation on a uniform grid
 *   (fastLPR_py/src/fastlpr/interp_optimized.py:60-215), OpenMP over points.
 *
 * Build: see oracle/build.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int64_t pmod(int64_t a, int64_t b) {
  int64_t r = a % b;
  return r < 0 ? r + b : r;
}

void oracle_spread(int d, int64_t n, const double* xmod, int C, const double* chans,
                   const int64_t* L, int msp, const double* tau, double* out) {
  double hx[3], four_tau[3];
  int64_t stride[3] = {1, 1, 1};
  for (int a = 0; a < d; ++a) {
    hx[a] = 2.0 * M_PI / (double)L[a];
    four_tau[a] = 4.0 * tau[a];
  }
  for (int a = d - 2; a >= 0; --a) stride[a] = stride[a + 1] * L[a + 1];
  const int nt = 2 * msp + 1;
  int64_t total = 1;
  for (int a = 0; a < d; ++a) total *= L[a];
  /* accumulate channel-innermost (one cache line per tap), transpose at the end */
  double* acc = (double*)calloc((size_t)total * C, sizeof(double));
  for (int64_t i = 0; i < n; ++i) {
    int64_t m[3] = {0, 0, 0};
    double ex[3][32];
    int64_t ix[3][32];
    for (int a = 0; a < d; ++a) {
      double k = xmod[i * d + a];
      m[a] = (int64_t)nearbyint(k / hx[a]);  /* default rounding mode: half to even */
      for (int j = 0; j < nt; ++j) {
        int64_t mj = m[a] + j - msp;
        double diff = k - hx[a] * (double)mj;
        ex[a][j] = diff * diff / four_tau[a];
        ix[a][j] = pmod(mj, L[a]) * stride[a];
      }
    }
    const double* v = chans + i * C;
    if (d == 1) {
      for (int j0 = 0; j0 < nt; ++j0) {
        double w = exp(-(ex[0][j0]));
        int64_t id = ix[0][j0];
        for (int c = 0; c < C; ++c) acc[id * C + c] += v[c] * w;
      }
    } else if (d == 2) {
      for (int j0 = 0; j0 < nt; ++j0)
        for (int j1 = 0; j1 < nt; ++j1) {
          double w = exp(-(ex[0][j0] + ex[1][j1]));
          int64_t id = ix[0][j0] + ix[1][j1];
          for (int c = 0; c < C; ++c) acc[id * C + c] += v[c] * w;
        }
    } else {
      for (int j0 = 0; j0 < nt; ++j0)
        for (int j1 = 0; j1 < nt; ++j1)
          for (int j2 = 0; j2 < nt; ++j2) {
            double w = exp(-(ex[0][j0] + ex[1][j1] + ex[2][j2]));
            int64_t id = ix[0][j0] + ix[1][j1] + ix[2][j2];
            for (int c = 0; c < C; ++c) acc[id * C + c] += v[c] * w;
          }
    }
  }
  for (int64_t id = 0; id < total; ++id)
    for (int c = 0; c < C; ++c) out[c * total + id] += acc[id * C + c];
  free(acc);
}

/* values: (M, K) row-major with M = prod G; out: (n, K). ax: {x0, dx} per axis. */
void oracle_interp(int d, int64_t n, const double* pts, const int64_t* G, const double* ax,
                   int64_t K, const double* values, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t ix[3] = {0, 0, 0};
    double fr[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) {
      double t = (pts[i * d + a] - ax[2 * a]) / ax[2 * a + 1];
      if (t < 0) {
        ix[a] = 0;
        fr[a] = 0.0;
      } else if (t >= (double)(G[a] - 1)) {
        ix[a] = G[a] - 2;
        fr[a] = 1.0;
      } else {
        ix[a] = (int64_t)t;
        fr[a] = t - (double)ix[a];
      }
    }
    double* o = out + i * K;
    for (int64_t k = 0; k < K; ++k) o[k] = 0.0;
    for (int c = 0; c < (1 << d); ++c) {
      int64_t idx = 0;
      double w = 1.0;
      for (int a = 0; a < d; ++a) {
        int bit = (c >> (d - 1 - a)) & 1;
        idx = idx * G[a] + ix[a] + bit;
        w *= bit ? fr[a] : 1.0 - fr[a];
      }
      const double* v = values + idx * K;
      for (int64_t k = 0; k < K; ++k) o[k] += w * v[k];
    }
  }
}
