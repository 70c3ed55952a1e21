// GCV, DoF and the 1-SE bandwidth choice on the device, and the gather of
// the chosen bandwidth's fitted grid: the output stage of a fit can then be
// enqueued (or captured in a CUDA graph) without waiting for the host.
//
// Same arithmetic, in the same order, as the host restatement of
// regression.py:280-471 (compute_gcv), regression.py:1276-1354 (Hutchinson
// DoF) and api.py:73-164 (1-SE rule): sums over the probes run sequentially
// in probe order like numpy's reductions over the leading axis of an
// (R, H) array, standard deviations are two-pass with ddof = 1.
#include <cmath>

#include "common.cuh"

namespace flpr {
namespace {

struct GcvArgs {
  int H, ny, R, dual, cplx, agg;  // agg: 0 first, 1 average, 2 sum
  double n, dstd;
};

__device__ __forceinline__ double clip_to(double v, double hi) {
  return v < 0.0 ? 0.0 : (v > hi ? hi : v);
}

// One block: thread per bandwidth for the scores, thread 0 for the choice.
// out: [gcv_m (H), gcv_sd (H), dof (H), dof_se (H)]; sel: chosen index or -1
// when no score is finite.
__global__ void gcv_select_kernel(GcvArgs a, const double* __restrict__ packed,
                                  const double* __restrict__ hsum, double* __restrict__ out,
                                  int* __restrict__ sel) {
  const int H = a.H, ny = a.ny, R = a.R;
  const int Cv = ny + R;
  const int Rm = R > 1 ? R : 1;
  const double n = a.n;
  const int dy = a.cplx ? ny / 2 : ny;
  for (int h = threadIdx.x; h < H; h += blockDim.x) {
    // RSS per response column
    double rss[FLPR_MAX_CHANNELS];
    for (int c = 0; c < ny; ++c) {
      double v;
      if (a.dual) {
        const double sq = packed[c], dot = packed[Cv + (int64_t)c * H + h];
        const double quad = packed[Cv + (int64_t)Cv * H + (int64_t)h * ny + c];
        v = sq - 2.0 * dot + quad;
      } else {
        v = packed[(int64_t)h * ny + c];
      }
      rss[c] = v;
    }
    if (a.cplx)
      for (int j = 0; j < dy; ++j) rss[j] = rss[2 * j] + rss[2 * j + 1];
    double dof = 0.0, dof_se = 0.0, pen_std = 0.0, pen_mean = 0.0;
    bool have_pen = false;
    {
      double tr[FLPR_MAX_CHANNELS];
      for (int r = 0; r < R; ++r) {
        double pdot, pp;
        if (a.dual) {
          pdot = packed[Cv + (int64_t)(ny + r) * H + h];
          pp = packed[ny + r];
        } else {
          pdot = packed[(int64_t)H * ny + (int64_t)r * H + h];
          pp = packed[(int64_t)H * ny + (int64_t)Rm * H + r];
        }
        double t = n * (pdot / pp);
        if (isnan(t)) t = n;
        tr[r] = clip_to(t, n);
      }
      double s = 0.0;
      for (int r = 0; r < R; ++r) s += tr[r];
      dof = s / (double)R;
      if (R > 1) {
        double q = 0.0;
        for (int r = 0; r < R; ++r) q += (tr[r] - dof) * (tr[r] - dof);
        dof_se = sqrt(q / (double)(R - 1)) / sqrt((double)R);
        double pen[FLPR_MAX_CHANNELS], pdc[FLPR_MAX_CHANNELS];
        for (int r = 0; r < R; ++r) {
          double pd = 1.0 - tr[r] / n;
          if (a.cplx) pd = 2.0 * pd - 1.0;
          pdc[r] = clip_to(pd, 1.0);
          const double mx = pdc[r] > 0.01 ? pdc[r] : 0.01;
          pen[r] = 1.0 / (mx * mx);
        }
        double ps = 0.0;
        for (int r = 0; r < R; ++r) ps += pen[r];
        pen_mean = ps / (double)R;
        double pq = 0.0;
        for (int r = 0; r < R; ++r) pq += (pen[r] - pen_mean) * (pen[r] - pen_mean);
        pen_std = sqrt(pq / (double)(R - 1));
        have_pen = true;
        if (a.cplx) {
          double cs = 0.0;
          for (int r = 0; r < R; ++r) cs += pdc[r];
          dof = n * (1.0 - cs / (double)R);
        }
      }
    }
    double pen_v;
    if (have_pen) {
      pen_v = pen_mean;
    } else {
      double pdv = clip_to(1.0 - dof / n, 1.0);
      pdv = pdv > 0.01 ? pdv : 0.01;
      pen_v = 1.0 / (pdv * pdv);
    }
    double sc, ms;
    if (a.agg == 0) {
      ms = rss[0] / n;
      sc = ms * pen_v;
    } else {
      double gs = 0.0, mss = 0.0;
      for (int j = 0; j < dy; ++j) {
        const double mj = rss[j] / n;
        gs += mj * pen_v;
        mss += mj;
      }
      sc = a.agg == 1 ? gs / (double)dy : gs;
      ms = a.agg == 1 ? mss / (double)dy : mss;
    }
    out[h] = sc;
    out[H + h] = pen_std > 0.0 ? ms * pen_std : 0.0;
    out[2 * H + h] = dof;
    out[3 * H + h] = dof_se;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double* vs = out;
    const double* ve = out + H;
    int b = -1;
    for (int h = 0; h < H; ++h)
      if (isfinite(vs[h]) && (b < 0 || vs[h] < vs[b])) b = h;
    int best = b;
    if (b >= 0) {
      const double thr = vs[b] + a.dstd * ve[b];
      double smax = -INFINITY;
      for (int h = 0; h < H; ++h)
        if (isfinite(vs[h]) && vs[h] <= thr && hsum[h] > smax) smax = hsum[h];
      int pick = -1;
      for (int h = 0; h < H; ++h)
        if (isfinite(vs[h]) && vs[h] <= thr && hsum[h] == smax && (pick < 0 || vs[h] < vs[pick]))
          pick = h;
      if (pick >= 0) best = pick;
    }
    *sel = best;
  }
}

// gv (ny, M) = m[sel][:, :ny] transposed; s0 (M) = S[0][sel] (as float64).
template <typename SReal>
__global__ void select_grid_kernel(int64_t M, int ny, int mstride, int H,
                                   const double* __restrict__ m, const SReal* __restrict__ S,
                                   const int* __restrict__ sel, double* __restrict__ gv,
                                   double* __restrict__ s0) {
  const int s = *sel;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (s < 0 || s >= H) {
      for (int c = 0; c < ny; ++c) gv[(int64_t)c * M + t] = NAN;
      s0[t] = NAN;
      continue;
    }
    const double* ms = m + ((int64_t)s * M + t) * mstride;
    for (int c = 0; c < ny; ++c) gv[(int64_t)c * M + t] = ms[c];
    s0[t] = (double)S[(int64_t)s * M + t];
  }
}

}  // namespace
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_gcv_select(int H, int ny, int R, int dual, int y_complex, int agg, double n, double dstd,
                    const double* d_packed, const double* d_hsum, double* d_out, int* d_sel,
                    void* stream) {
  FLPR_CHECK_ARG(H >= 1 && ny >= 1 && R >= 0 && ny + R <= FLPR_MAX_CHANNELS,
                 "gcv_select: H=%d ny=%d R=%d", H, ny, R);
  FLPR_CHECK_ARG(!y_complex || ny % 2 == 0, "gcv_select: complex needs pairs of channels");
  FLPR_CHECK_ARG(agg >= 0 && agg <= 2, "gcv_select: agg=%d", agg);
  FLPR_CHECK_ARG(n >= 1.0, "gcv_select: n=%g", n);
  FLPR_CHECK_ARG(d_packed && d_hsum && d_out && d_sel, "gcv_select: null pointer");
  GcvArgs a{H, ny, R, dual ? 1 : 0, y_complex ? 1 : 0, agg, n, dstd};
  gcv_select_kernel<<<1, 256, 0, as_stream(stream)>>>(a, d_packed, d_hsum, d_out, d_sel);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_select_grid(int64_t M, int ny, int mstride, int H, const double* d_m, const void* d_S,
                     int s_prec, const int* d_sel, double* d_gv, double* d_s0, void* stream) {
  FLPR_CHECK_ARG(M >= 1 && ny >= 1 && mstride >= ny && H >= 1,
                 "select_grid: M=%lld ny=%d mstride=%d H=%d", (long long)M, ny, mstride, H);
  FLPR_CHECK_ARG(d_m && d_S && d_sel && d_gv && d_s0, "select_grid: null pointer");
  int64_t b = (M + 255) / 256;
  if (b > 8 * sm_count()) b = 8 * sm_count();
  cudaStream_t s = as_stream(stream);
  if (s_prec == FLPR_PREC_F32)
    select_grid_kernel<float><<<(int)b, 256, 0, s>>>(M, ny, mstride, H, d_m,
                                                     static_cast<const float*>(d_S), d_sel, d_gv,
                                                     d_s0);
  else
    select_grid_kernel<double><<<(int)b, 256, 0, s>>>(M, ny, mstride, H, d_m,
                                                      static_cast<const double*>(d_S), d_sel,
                                                      d_gv, d_s0);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
