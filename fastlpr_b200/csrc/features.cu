// Binned moment sums of a data set, the input summary of the bandwidth
// proposal network: on a grid of 4096 cells spanning [min, max] of every
// axis (4096 bins in 1-D, 64 x 64 in 2-D), the count, sum y and sum y^2 of
// the points in each cell.
#include "common.cuh"

#include <cuda_bf16.h>

namespace flpr {
namespace {

constexpr int kFeatCells = 4096;
__host__ __device__ constexpr int feat_bins(int d) { return d == 1 ? 4096 : 64; }

// grid-stride over the points; per-block float histogram in shared memory,
// flushed to the FP64 output with one atomic per non-zero cell
__global__ void bin_moments_kernel(int d, int64_t n, const double* __restrict__ x,
                                   const double* __restrict__ y, const double* __restrict__ stats,
                                   double* __restrict__ out) {
  extern __shared__ float hist[];  // 3 x cells
  const int cells = kFeatCells, bins = feat_bins(d);
  for (int i = threadIdx.x; i < 3 * cells; i += blockDim.x) hist[i] = 0.0f;
  __syncthreads();
  double lo[2], scale[2];
  for (int a = 0; a < d; ++a) {
    lo[a] = stats[a];
    const double span = stats[d + a] - stats[a];
    scale[a] = span > 0.0 ? (double)bins / span : 0.0;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int cell = 0;
    for (int a = 0; a < d; ++a) {
      int b = (int)floor((x[i * d + a] - lo[a]) * scale[a]);
      b = b < 0 ? 0 : (b >= bins ? bins - 1 : b);
      cell = cell * bins + b;
    }
    const float v = (float)y[i];
    atomicAdd(&hist[cell], 1.0f);
    atomicAdd(&hist[cells + cell], v);
    atomicAdd(&hist[2 * cells + cell], v * v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * cells; i += blockDim.x)
    if (hist[i] != 0.0f) atomicAdd(&out[i], (double)hist[i]);
}

// ---- feature vector of the proposal network, on the device -------------
// One CTA per data set turns its binned sums (3 x 4096: count, sum y,
// sum y^2) into the FEATURE_DIM = 416 summary that learned.summarize forms
// on the host (same formulas and layout), standardises it with the
// network's feature mean / std and stores it as BF16, the network's input.
constexpr int kFeatDim = 416;
constexpr int kFeatThreads = 256;
constexpr int kLags = 12;

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = 0.0;
  for (int w = 0; w < kFeatThreads / 32; ++w) r += red[w];  // same order in every thread
  return r;
}

// marginal bin b of axis a of a 4096-cell field (64 cells per bin)
__device__ __forceinline__ double axis_bin(const double* f, int d, int a, int b) {
  double s = 0.0;
  if (d == 1 || a == 0) {
    for (int j = 0; j < 64; ++j) s += f[64 * b + j];
  } else {
    for (int i = 0; i < 64; ++i) s += f[64 * i + b];
  }
  return s;
}

__global__ void __launch_bounds__(kFeatThreads)
features_kernel(const double* __restrict__ bins, const int* __restrict__ meta,
                const float* __restrict__ fmean, const float* __restrict__ fstd,
                float* __restrict__ feat_out, __nv_bfloat16* __restrict__ x16) {
  extern __shared__ double sm[];
  double* cnt = sm;                 // 4096
  double* sz = cnt + kFeatCells;    // 4096: standardised sums, then cell means
  double* szz = sz + kFeatCells;    // 4096: standardised sums of squares, then 1/count
  __shared__ double red[kFeatThreads / 32];
  __shared__ double f[kFeatDim];
  const int prob = blockIdx.x;
  const int d = meta[3 * prob], order = meta[3 * prob + 1], n = meta[3 * prob + 2];
  const double* b = bins + (size_t)prob * 3 * kFeatCells;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < kFeatCells; i += kFeatThreads) {
    const double c = b[i], y1 = b[kFeatCells + i], y2 = b[2 * kFeatCells + i];
    cnt[i] = c;
    sz[i] = y1;
    szz[i] = y2;
    s0 += c;
    s1 += y1;
    s2 += y2;
  }
  for (int i = threadIdx.x; i < kFeatDim; i += kFeatThreads) f[i] = 0.0;
  const double N = fmax(block_sum_d(s0, red), 1.0);
  const double ybar = block_sum_d(s1, red) / N;
  const double var = fmax(block_sum_d(s2, red) / N - ybar * ybar, 0.0);
  const double sd = var > 0.0 ? __dsqrt_rn(var) : 1.0;
  // standardised sums per cell; within-cell variance over cells with >= 2 points
  double wnum = 0.0, wden = 0.0;
  for (int i = threadIdx.x; i < kFeatCells; i += kFeatThreads) {
    const double c = cnt[i], y1 = sz[i], y2 = szz[i];
    const double a1 = (y1 - c * ybar) / sd;
    const double a2 = (y2 - 2.0 * ybar * y1 + c * ybar * ybar) / (sd * sd);
    sz[i] = a1;
    szz[i] = a2;
    if (c >= 2.0) {
      wnum += a2 - a1 * a1 / c;
      wden += c - 1.0;
    }
  }
  __syncthreads();
  // per-axis 64-bin marginals of the count, mean and mean square
  for (int t = threadIdx.x; t < 64 * d; t += kFeatThreads) {
    const int a = t / 64, bb = t % 64;
    const double c = axis_bin(cnt, d, a, bb);
    const double m1 = axis_bin(sz, d, a, bb), m2 = axis_bin(szz, d, a, bb);
    f[192 * a + bb] = 64.0 * c / N;
    f[192 * a + 64 + bb] = c > 0.0 ? m1 / fmax(c, 1.0) : 0.0;
    f[192 * a + 128 + bb] = c > 0.0 ? m2 / fmax(c, 1.0) : 0.0;
  }
  const double wn = block_sum_d(wnum, red), wd = block_sum_d(wden, red);
  const double within = fmax(wd > 0.0 ? wn / wd : 0.0, 0.0);
  // cell means and inverse counts (NaN for empty cells)
  for (int i = threadIdx.x; i < kFeatCells; i += kFeatThreads) {
    const double c = cnt[i];
    const double mu = c > 0.0 ? sz[i] / fmax(c, 1.0) : NAN;
    const double inv = c > 0.0 ? 1.0 / fmax(c, 1.0) : NAN;
    sz[i] = mu;
    szz[i] = inv;
  }
  __syncthreads();
  // lag roughness: mean squared difference of the cell means at lag 2^k of
  // the 4096-cell span (per axis of the 64 x 64 field in 2-D), raw and less
  // the expected noise; the mean over the axes that have a valid pair
  for (int k = 0; k < kLags; ++k) {
    int lag = 1 << k;
    if (d == 2) {
      if (lag < 64) continue;
      lag /= 64;
    }
    double raw_sum = 0.0, cor_sum = 0.0, naxes = 0.0;
    for (int a = 0; a < d; ++a) {
      const int ext = d == 1 ? kFeatCells : 64;
      const int npairs = d == 1 ? ext - lag : (ext - lag) * 64;
      double sr = 0.0, sn = 0.0, sc = 0.0;
      for (int q = threadIdx.x; q < npairs; q += kFeatThreads) {
        int i0, i1;
        if (d == 1) {
          i0 = q;
          i1 = q + lag;
        } else if (a == 0) {  // rows: (r, c) and (r + lag, c)
          i0 = q;
          i1 = q + 64 * lag;
        } else {              // columns: (r, c) and (r, c + lag)
          const int r = q / (64 - lag), c = q % (64 - lag);
          i0 = 64 * r + c;
          i1 = i0 + lag;
        }
        const double df = sz[i1] - sz[i0];
        if (isfinite(df)) {
          sr += df * df;
          sn += within * (szz[i1] + szz[i0]);
          sc += 1.0;
        }
      }
      sr = block_sum_d(sr, red);
      sn = block_sum_d(sn, red);
      sc = block_sum_d(sc, red);
      if (sc > 0.0) {
        const double r = sr / sc;
        raw_sum += r;
        cor_sum += r - sn / sc;
        naxes += 1.0;
      }
    }
    if (threadIdx.x == 0 && naxes > 0.0) {
      f[384 + k] = raw_sum / naxes;
      f[384 + kLags + k] = cor_sum / naxes;
    }
  }
  if (threadIdx.x == 0) {
    f[408] = within;
    f[409] = log10(within + 1e-6) / 3.0;
    f[410] = log10(fmax((double)n, 1.0)) / 6.0;
    f[411 + order] = 1.0;
    f[414 + (d - 1)] = 1.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kFeatDim; i += kFeatThreads) {
    const float v = (float)f[i];
    if (feat_out) feat_out[(size_t)prob * kFeatDim + i] = v;
    const float z = __fdiv_rn(__fsub_rn(v, fmean[i]), fstd[i]);
    x16[(size_t)prob * kFeatDim + i] = __float2bfloat16_rn(z);
  }
}

// Window of `refine` neighbouring bandwidths around the network's proposal
// (learned.refine_window): t = clip(raw * t_scale + t_center, 0, ngrid - 1)
// on the canonical grid, target log h interpolated there, the nearest entry
// c of the problem's own log-h list (first one on ties) and the window start
// clip(c - refine / 2, 0, nlist - refine).  No fused multiply-adds, so the
// arithmetic is the host's.
__global__ void window_kernel(int B, const float* __restrict__ raw, double t_scale,
                              double t_center, int ngrid, const double* __restrict__ loggrid,
                              int lmax, const int* __restrict__ nlist,
                              const double* __restrict__ logh, int refine,
                              int* __restrict__ lo_out, double* __restrict__ t_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= B) return;
  double t = __dadd_rn(__dmul_rn((double)raw[p], t_scale), t_center);
  if (t_out) t_out[p] = t;
  t = fmin(fmax(t, 0.0), (double)(ngrid - 1));
  const int i0 = (int)floor(t);
  const int i1 = min(i0 + 1, ngrid - 1);
  const double target =
      __dadd_rn(loggrid[i0], __dmul_rn(__dsub_rn(t, (double)i0), __dsub_rn(loggrid[i1], loggrid[i0])));
  const int nl = nlist[p];
  const double* lh = logh + (size_t)p * lmax;
  int c = 0;
  double best = fabs(__dsub_rn(lh[0], target));
  for (int i = 1; i < nl; ++i) {
    const double e = fabs(__dsub_rn(lh[i], target));
    if (e < best) {
      best = e;
      c = i;
    }
  }
  lo_out[p] = min(max(c - refine / 2, 0), nl - refine);
}

// rows [start, start + rows) of a row-major array, start read on the device
__global__ void copy_rows_kernel(const unsigned long long* __restrict__ src,
                                 unsigned long long* __restrict__ dst, int64_t row_words,
                                 int rows, const int* __restrict__ d_start) {
  const int64_t total = row_words * rows;
  const int64_t off = (int64_t)(*d_start) * row_words;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[off + i];
}

}  // namespace
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_bin_moments(int d, int64_t n, const double* d_x, const double* d_y, const double* d_stats,
                     double* d_out, void* stream) {
  FLPR_CHECK_ARG(d == 1 || d == 2, "bin_moments: d=%d (1 or 2)", d);
  FLPR_CHECK_ARG(n >= 1, "bin_moments: n=%lld", (long long)n);
  const int cells = kFeatCells;
  cudaStream_t s = as_stream(stream);
  FLPR_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * 3 * cells, s));
  const size_t smem = sizeof(float) * 3 * cells;
  int nb = (int)((n + 1023) / 1024);
  if (nb > 2 * sm_count()) nb = 2 * sm_count();
  if (nb < 1) nb = 1;
  bin_moments_kernel<<<nb, 256, smem, s>>>(d, n, d_x, d_y, d_stats, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_learned_features(int B, const double* d_bins, const int* d_meta, const float* d_fmean,
                          const float* d_fstd, float* d_feat, void* d_x16, void* stream) {
  FLPR_CHECK_ARG(B >= 1, "learned_features: B=%d", B);
  FLPR_CHECK_ARG(d_bins && d_meta && d_fmean && d_fstd && d_x16,
                 "learned_features: null pointer");
  const size_t smem = sizeof(double) * 3 * kFeatCells;
  FLPR_CUDA(raise_dyn_smem(features_kernel, smem));
  features_kernel<<<B, kFeatThreads, smem, as_stream(stream)>>>(
      d_bins, d_meta, d_fmean, d_fstd, d_feat, static_cast<__nv_bfloat16*>(d_x16));
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_learned_window(int B, const float* d_raw, double t_scale, double t_center, int ngrid,
                        const double* d_loggrid, int lmax, const int* d_nlist,
                        const double* d_logh, int refine, int* d_lo, double* d_t,
                        void* stream) {
  FLPR_CHECK_ARG(B >= 1 && ngrid >= 1 && refine >= 1 && lmax >= refine,
                 "learned_window: B=%d ngrid=%d lmax=%d refine=%d", B, ngrid, lmax, refine);
  FLPR_CHECK_ARG(d_raw && d_loggrid && d_nlist && d_logh && d_lo, "learned_window: null pointer");
  window_kernel<<<(B + 127) / 128, 128, 0, as_stream(stream)>>>(
      B, d_raw, t_scale, t_center, ngrid, d_loggrid, lmax, d_nlist, d_logh, refine, d_lo, d_t);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_copy_rows(const void* d_src, void* d_dst, int64_t row_bytes, int rows,
                   const int* d_start, void* stream) {
  FLPR_CHECK_ARG(row_bytes > 0 && row_bytes % 8 == 0 && rows >= 1,
                 "copy_rows: row_bytes=%lld rows=%d", (long long)row_bytes, rows);
  FLPR_CHECK_ARG(d_src && d_dst && d_start, "copy_rows: null pointer");
  const int64_t words = row_bytes / 8 * rows;
  int nb = (int)((words + 255) / 256);
  if (nb > 4 * sm_count()) nb = 4 * sm_count();
  copy_rows_kernel<<<nb, 256, 0, as_stream(stream)>>>(
      static_cast<const unsigned long long*>(d_src), static_cast<unsigned long long*>(d_dst),
      row_bytes / 8, rows, d_start);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
