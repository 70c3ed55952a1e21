// Not-a-knot cubic spline interpolation of grid values at the data points:
// the 'cubic' GCV/DoF interpolation of the reference (api.py:594-600,
// api.py:651-657, regression.py:1015-1020), which is scipy's
// RegularGridInterpolator(method='cubic', fill_value=None): per axis the
// knots t = [x0]*4 + x[2:-2] + [x_end]*4, coefficients from the tensor
// collocation system, end polynomial pieces extended beyond the grid.
//
// Two steps:
//  * spline_prefilter: the tensor collocation matrix is the Kronecker product
//    of per-axis banded matrices (bandwidth 3 either side); its LU factors
//    (no pivoting: B-spline collocation matrices are totally positive) come
//    from the host, one line of grid values per thread is solved in place,
//    axis by axis.
//  * spline_reduce / spline_eval: the 4 non-zero B-splines per axis at each
//    point (Cox-de Boor recursion, triangular form of Piegl and Tiller, The
//    NURBS Book, A2.2) weight the 4^d coefficients around it.
#include "common.cuh"

namespace flpr {
namespace spl {

constexpr int kMaxRed = 32;  // values reduced per (point, bandwidth)
constexpr int kLuCols = 7;   // l3 l2 l1 1/u0 u1 u2 u3 per row

struct Geom {
  int d;
  int G[3];
  int64_t M;
  const double* ax[3];  // device: raw grid axes (strictly increasing)
};

struct Cols {
  const double* col[kMaxRed];
};

__device__ __forceinline__ double knot(const double* __restrict__ ax, int G, int j) {
  return j <= 3 ? ax[0] : (j >= G ? ax[G - 1] : ax[j - 2]);
}

// Weights of the B-splines first..first+3 at x (first = span - 3).
__device__ __forceinline__ void bspline4(const double* __restrict__ ax, int G, double x, int* first,
                                         double w[4]) {
  int lo = -1, hi = G;  // largest j with ax[j] <= x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (ax[mid] <= x) lo = mid; else hi = mid;
  }
  int l = lo + 2;
  l = l < 3 ? 3 : (l > G - 1 ? G - 1 : l);
  double left[4], right[4];
  w[0] = 1.0;
#pragma unroll
  for (int j = 1; j <= 3; ++j) {
    left[j] = x - knot(ax, G, l + 1 - j);
    right[j] = knot(ax, G, l + j) - x;
    double saved = 0.0;
#pragma unroll
    for (int r = 0; r < j; ++r) {
      const double temp = w[r] / (right[r + 1] + left[j - r]);
      w[r] = saved + right[r + 1] * temp;
      saved = left[j - r] * temp;
    }
    w[j] = saved;
  }
  *first = l - 3;
}

template <int D>
struct PointTaps {
  int first[D];
  double w[D][4];
};

template <int D>
__device__ __forceinline__ void point_taps(const Geom& g, const double* __restrict__ x, int64_t i,
                                           PointTaps<D>& pt) {
#pragma unroll
  for (int a = 0; a < D; ++a) bspline4(g.ax[a], g.G[a], x[i * D + a], &pt.first[a], pt.w[a]);
}

// sum_taps w * v[idx * C + c]
template <int D>
__device__ __forceinline__ double tap_sum(const Geom& g, const PointTaps<D>& pt,
                                          const double* __restrict__ v, int C, int c) {
  double s = 0.0;
  if (D == 1) {
#pragma unroll
    for (int a0 = 0; a0 < 4; ++a0) s += pt.w[0][a0] * v[(int64_t)(pt.first[0] + a0) * C + c];
  } else if (D == 2) {
#pragma unroll
    for (int a0 = 0; a0 < 4; ++a0) {
      const int64_t r0 = (int64_t)(pt.first[0] + a0) * g.G[1];
      double s1 = 0.0;
#pragma unroll
      for (int a1 = 0; a1 < 4; ++a1) s1 += pt.w[1][a1] * v[(r0 + pt.first[1] + a1) * C + c];
      s += pt.w[0][a0] * s1;
    }
  } else {
#pragma unroll
    for (int a0 = 0; a0 < 4; ++a0) {
      double s1 = 0.0;
#pragma unroll
      for (int a1 = 0; a1 < 4; ++a1) {
        const int64_t r01 = ((int64_t)(pt.first[0] + a0) * g.G[1] + pt.first[1] + a1) * g.G[2];
        double s2 = 0.0;
#pragma unroll
        for (int a2 = 0; a2 < 4; ++a2) s2 += pt.w[2][a2] * v[(r01 + pt.first[2] + a2) * C + c];
        s1 += pt.w[1][a1] * s2;
      }
      s += pt.w[0][a0] * s1;
    }
  }
  return s;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
  return r;  // valid in thread 0
}

// One line per thread: forward substitution with L (unit diagonal), back
// substitution with U.  Lines are (block, q) with q fastest, so neighbouring
// threads touch neighbouring addresses except along the innermost axis.
__global__ void prefilter_kernel(int64_t nlines, int G, int64_t stride,
                                 const double* __restrict__ lu, double* __restrict__ v) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nlines;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t blk = t / stride, q = t - blk * stride;
    double* p = v + blk * (int64_t)G * stride + q;
    double y1 = 0.0, y2 = 0.0, y3 = 0.0;
    for (int i = 0; i < G; ++i) {
      const double* f = lu + (int64_t)kLuCols * i;
      const double yi = p[i * stride] - f[2] * y1 - f[1] * y2 - f[0] * y3;
      p[i * stride] = yi;
      y3 = y2;
      y2 = y1;
      y1 = yi;
    }
    double x1 = 0.0, x2 = 0.0, x3 = 0.0;
    for (int i = G - 1; i >= 0; --i) {
      const double* f = lu + (int64_t)kLuCols * i;
      const double xi = (p[i * stride] - f[4] * x1 - f[5] * x2 - f[6] * x3) * f[3];
      p[i * stride] = xi;
      x3 = x2;
      x2 = x1;
      x1 = xi;
    }
  }
}

// blockIdx.y = bandwidth.  coef: (H, M, C) with C = ny + R.
template <int D>
__global__ void reduce_kernel(Geom g, int64_t n, const double* __restrict__ x, int H, int ny,
                              int R, const double* __restrict__ coef, Cols yc, Cols pc,
                              double* __restrict__ rss, double* __restrict__ pdot) {
  __shared__ double sh[32];
  const int h = blockIdx.y;
  const int C = ny + R;
  double acc[kMaxRed];
#pragma unroll
  for (int c = 0; c < kMaxRed; ++c) acc[c] = 0.0;
  const double* ch = coef + (int64_t)h * g.M * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    PointTaps<D> pt;
    point_taps<D>(g, x, i, pt);
#pragma unroll
    for (int c = 0; c < kMaxRed; ++c) {
      if (c < C) {
        const double v = tap_sum<D>(g, pt, ch, C, c);
        if (c < ny) {
          const double r = yc.col[c][i] - v;
          acc[c] += r * r;
        } else {
          acc[c] += pc.col[c - ny][i] * v;
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < kMaxRed; ++c) {
    if (c < C) {
      const double s = block_sum(acc[c], sh);
      if (threadIdx.x == 0) {
        if (c < ny) atomicAdd(&rss[h * ny + c], s);
        else atomicAdd(&pdot[(c - ny) * H + h], s);
      }
    }
  }
}

__global__ void probe_norm_kernel(int64_t n, int R, Cols pc, double* __restrict__ pp) {
  __shared__ double sh[32];
  for (int r = 0; r < R; ++r) {
    double a = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
      const double v = pc.col[r][i];
      a += v * v;
    }
    const double s = block_sum(a, sh);
    if (threadIdx.x == 0) atomicAdd(&pp[r], s);
  }
}

// coef: (nval, M) -> out (nval, n)
template <int D>
__global__ void eval_kernel(Geom g, int64_t n, const double* __restrict__ x, int nval,
                            const double* __restrict__ coef, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    PointTaps<D> pt;
    point_taps<D>(g, x, i, pt);
    for (int v = 0; v < nval; ++v)
      out[(int64_t)v * n + i] = tap_sum<D>(g, pt, coef + (int64_t)v * g.M, 1, 0);
  }
}

static int make_geom(Geom& g, int d, const double* d_axes, const int* h_G) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "spline: d=%d not in [1,3]", d);
  FLPR_CHECK_ARG(d_axes != nullptr, "spline: axes pointer is null");
  memset(&g, 0, sizeof(g));
  g.d = d;
  g.M = 1;
  int64_t off = 0;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(h_G[a] >= 4 && h_G[a] <= (1 << 20),
                   "spline: G[%d]=%d (cubic needs at least 4 grid points per axis)", a, h_G[a]);
    g.G[a] = h_G[a];
    g.ax[a] = d_axes + off;
    off += h_G[a];
    g.M *= h_G[a];
  }
  return FLPR_OK;
}

static int point_blocks(int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = 4 * (int64_t)sm_count();
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace spl
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_spline_prefilter(int d, const int* h_G, int64_t outer, int inner, const double* d_lu,
                          double* d_vals, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "spline_prefilter: d=%d not in [1,3]", d);
  FLPR_CHECK_ARG(outer >= 1 && inner >= 1, "spline_prefilter: outer=%lld inner=%d",
                 (long long)outer, inner);
  FLPR_CHECK_ARG(d_lu != nullptr && d_vals != nullptr, "spline_prefilter: null pointer");
  int64_t M = 1;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(h_G[a] >= 4, "spline_prefilter: G[%d]=%d < 4", a, h_G[a]);
    M *= h_G[a];
  }
  cudaStream_t s = as_stream(stream);
  const int64_t total = outer * M * inner;
  int64_t lu_off = 0;
  for (int a = 0; a < d; ++a) {
    int64_t stride = inner;
    for (int b = a + 1; b < d; ++b) stride *= h_G[b];
    const int64_t nlines = total / h_G[a];
    int nb = (int)((nlines + 127) / 128);
    if (nb > 16 * sm_count()) nb = 16 * sm_count();
    spl::prefilter_kernel<<<nb, 128, 0, s>>>(nlines, h_G[a], stride, d_lu + lu_off, d_vals);
    FLPR_LAUNCH_CHECK();
    lu_off += (int64_t)spl::kLuCols * h_G[a];
  }
  return FLPR_OK;
}

int flpr_spline_reduce(int d, int64_t n, const double* d_x, const double* d_axes, const int* h_G,
                       int H, int ny, int R, const double* d_coef, const double* const* h_ycols,
                       const double* const* h_pcols, double* d_rss, double* d_pdot, double* d_pp,
                       void* stream) {
  spl::Geom g;
  FLPR_TRY(spl::make_geom(g, d, d_axes, h_G));
  FLPR_CHECK_ARG(n >= 1 && H >= 1 && ny >= 0 && R >= 0 && ny + R >= 1 && ny + R <= spl::kMaxRed,
                 "spline_reduce: n=%lld H=%d ny=%d R=%d", (long long)n, H, ny, R);
  cudaStream_t s = as_stream(stream);
  spl::Cols yc, pc;
  memset(&yc, 0, sizeof(yc));
  memset(&pc, 0, sizeof(pc));
  for (int c = 0; c < ny; ++c) yc.col[c] = h_ycols[c];
  for (int r = 0; r < R; ++r) pc.col[r] = h_pcols[r];
  if (ny) FLPR_CUDA(cudaMemsetAsync(d_rss, 0, sizeof(double) * H * ny, s));
  if (R) {
    FLPR_CUDA(cudaMemsetAsync(d_pdot, 0, sizeof(double) * H * R, s));
    FLPR_CUDA(cudaMemsetAsync(d_pp, 0, sizeof(double) * R, s));
  }
  int per_h = (spl::point_blocks(n) + H - 1) / H;
  if (per_h < 8) per_h = 8;
  dim3 grid(per_h, H);
  if (d == 1)
    spl::reduce_kernel<1><<<grid, 256, 0, s>>>(g, n, d_x, H, ny, R, d_coef, yc, pc, d_rss, d_pdot);
  else if (d == 2)
    spl::reduce_kernel<2><<<grid, 256, 0, s>>>(g, n, d_x, H, ny, R, d_coef, yc, pc, d_rss, d_pdot);
  else
    spl::reduce_kernel<3><<<grid, 256, 0, s>>>(g, n, d_x, H, ny, R, d_coef, yc, pc, d_rss, d_pdot);
  FLPR_LAUNCH_CHECK();
  if (R) {
    spl::probe_norm_kernel<<<spl::point_blocks(n), 256, 0, s>>>(n, R, pc, d_pp);
    FLPR_LAUNCH_CHECK();
  }
  return FLPR_OK;
}

int flpr_spline_eval(int d, int64_t n, const double* d_x, const double* d_axes, const int* h_G,
                     int nval, const double* d_coef, double* d_out, void* stream) {
  spl::Geom g;
  FLPR_TRY(spl::make_geom(g, d, d_axes, h_G));
  FLPR_CHECK_ARG(n >= 1 && nval >= 1, "spline_eval: n=%lld nval=%d", (long long)n, nval);
  cudaStream_t s = as_stream(stream);
  const int nb = spl::point_blocks(n);
  if (d == 1)
    spl::eval_kernel<1><<<nb, 256, 0, s>>>(g, n, d_x, nval, d_coef, d_out);
  else if (d == 2)
    spl::eval_kernel<2><<<nb, 256, 0, s>>>(g, n, d_x, nval, d_coef, d_out);
  else
    spl::eval_kernel<3><<<nb, 256, 0, s>>>(g, n, d_x, nval, d_coef, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
