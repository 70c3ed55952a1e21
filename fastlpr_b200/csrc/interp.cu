// Grid -> point interpolation, GCV / Hutchinson reductions and KDE LCV.
#include "common.cuh"

namespace flpr {

constexpr int kMaxRed = 32;  // values reduced per (point, bandwidth)

struct InterpGeom {
  int d;
  int G[3];
  double x0[3], dx[3];
  int64_t M;
};

// Cell and fraction on one axis, clamped like interp_optimized.py:60-78.
__device__ __forceinline__ void axis_cell(double xi, double x0, double dx, int nx, int* ix,
                                          double* fr) {
  double t = (xi - x0) / dx;
  if (t < 0.0) {
    *ix = 0;
    *fr = 0.0;
  } else if (t >= (double)(nx - 1)) {
    *ix = nx - 2 < 0 ? 0 : nx - 2;
    *fr = 1.0;
  } else {
    int i = (int)t;
    *ix = i;
    *fr = t - (double)i;
  }
}

// Corner offsets/weights of the multilinear stencil of point i.
struct Stencil {
  int64_t base[8];
  double w[8];
  int ncorner;
};

__device__ __forceinline__ void make_stencil(const InterpGeom& g, const double* __restrict__ x,
                                             int64_t i, Stencil& st) {
  int ix[3] = {0, 0, 0};
  double fr[3] = {0, 0, 0};
  for (int a = 0; a < g.d; ++a) axis_cell(x[i * g.d + a], g.x0[a], g.dx[a], g.G[a], &ix[a], &fr[a]);
  st.ncorner = 1 << g.d;
  for (int c = 0; c < st.ncorner; ++c) {
    int64_t idx = 0;
    double w = 1.0;
    for (int a = 0; a < g.d; ++a) {
      int bit = (c >> (g.d - 1 - a)) & 1;
      int ia = ix[a] + bit;
      if (ia >= g.G[a]) ia = g.G[a] - 1;  // single-point axis
      idx = idx * g.G[a] + ia;
      w *= bit ? fr[a] : (1.0 - fr[a]);
    }
    st.base[c] = idx;
    st.w[c] = w;
  }
}

// The same stencil with the dimension fixed at compile time (corners held
// in registers): identical indices, weights and order.
template <int D>
struct StencilD {
  int64_t base[1 << D];
  double w[1 << D];
};

template <int D>
__device__ __forceinline__ void make_stencil_d(const InterpGeom& g, const double* __restrict__ x,
                                               int64_t i, StencilD<D>& st) {
  int ix[D];
  double fr[D];
#pragma unroll
  for (int a = 0; a < D; ++a) axis_cell(x[i * D + a], g.x0[a], g.dx[a], g.G[a], &ix[a], &fr[a]);
#pragma unroll
  for (int c = 0; c < (1 << D); ++c) {
    int64_t idx = 0;
    double w = 1.0;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const int bit = (c >> (D - 1 - a)) & 1;
      int ia = ix[a] + bit;
      if (ia >= g.G[a]) ia = g.G[a] - 1;  // single-point axis
      idx = idx * g.G[a] + ia;
      w *= bit ? fr[a] : (1.0 - fr[a]);
    }
    st.base[c] = idx;
    st.w[c] = w;
  }
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

struct ColPtrs {
  const double* col[kMaxRed];
};

// blockIdx.y = bandwidth.  m: (H, M, C) with C = ny + R.
__global__ void interp_reduce_kernel(InterpGeom g, int64_t n, const double* __restrict__ x, int H,
                                     int ny, int R, const double* __restrict__ m, ColPtrs yc,
                                     ColPtrs pc, double* __restrict__ rss,
                                     double* __restrict__ pdot) {
  __shared__ double sh[32];
  const int h = blockIdx.y;
  const int C = ny + R;
  double acc[kMaxRed];
#pragma unroll
  for (int c = 0; c < kMaxRed; ++c) acc[c] = 0.0;
  const double* mh = m + (int64_t)h * g.M * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Stencil st;
    make_stencil(g, x, i, st);
#pragma unroll
    for (int c = 0; c < kMaxRed; ++c) {
      if (c < C) {
        double v = 0.0;
        for (int k = 0; k < st.ncorner; ++k) v += st.w[k] * mh[st.base[k] * C + c];
        if (c < ny) {
          double r = yc.col[c][i] - v;
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
      double s = block_sum(acc[c], sh);
      if (threadIdx.x == 0) {
        if (c < ny) atomicAdd(&rss[h * ny + c], s);
        else atomicAdd(&pdot[(c - ny) * H + h], s);
      }
    }
  }
}

__global__ void probe_norm_kernel(int64_t n, int R, ColPtrs pc, double* __restrict__ pp) {
  __shared__ double sh[32];
  for (int r = 0; r < R; ++r) {
    double a = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
      double v = pc.col[r][i];
      a += v * v;
    }
    double s = block_sum(a, sh);
    if (threadIdx.x == 0) atomicAdd(&pp[r], s);
  }
}

// Edge-cell continuation on one axis (scipy's RegularGridInterpolator with
// fill_value=None): the cell index clamped to [0, nx - 2], the fraction not.
__device__ __forceinline__ void axis_cell_extrap(double xi, double x0, double dx, int nx, int* ix,
                                                 double* fr) {
  const double t = (xi - x0) / dx;
  int i = (int)floor(t);
  const int top = nx - 2 < 0 ? 0 : nx - 2;
  i = i < 0 ? 0 : (i > top ? top : i);
  *ix = i;
  *fr = t - (double)i;
}

template <bool kExtrap>
__global__ void interp_eval_kernel(InterpGeom g, int64_t n, const double* __restrict__ x, int nval,
                                   const double* __restrict__ vals, double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Stencil st;
    if (kExtrap) {
      int ix[3] = {0, 0, 0};
      double fr[3] = {0, 0, 0};
      for (int a = 0; a < g.d; ++a)
        axis_cell_extrap(x[i * g.d + a], g.x0[a], g.dx[a], g.G[a], &ix[a], &fr[a]);
      st.ncorner = 1 << g.d;
      for (int c = 0; c < st.ncorner; ++c) {
        int64_t idx = 0;
        double w = 1.0;
        for (int a = 0; a < g.d; ++a) {
          const int bit = (c >> (g.d - 1 - a)) & 1;
          int ia = ix[a] + bit;
          if (ia >= g.G[a]) ia = g.G[a] - 1;  // single-point axis
          idx = idx * g.G[a] + ia;
          w *= bit ? fr[a] : (1.0 - fr[a]);
        }
        st.base[c] = idx;
        st.w[c] = w;
      }
    } else {
      make_stencil(g, x, i, st);
    }
    for (int v = 0; v < nval; ++v) {
      const double* vv = vals + (int64_t)v * g.M;
      double r = 0.0;
      for (int k = 0; k < st.ncorner; ++k) r += st.w[k] * vv[st.base[k]];
      out[(int64_t)v * n + i] = r;
    }
  }
}

// ---- KDE -----------------------------------------------------------------
__global__ void plane_sum_kernel(int64_t M, const double* __restrict__ s, double* __restrict__ sums) {
  __shared__ double sh[32];
  const int h = blockIdx.y;
  const double* p = s + (int64_t)h * M;
  double a = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x)
    a += p[i];
  double t = block_sum(a, sh);
  if (threadIdx.x == 0) atomicAdd(&sums[h], t);
}

// f (H, M) and its bandwidth-fastest copy fT (M, H), through a 32 x 32 tile:
// grid (ceil(M / 32), ceil(H / 32)), block (32, 8).
__global__ void kde_normalize_kernel(int64_t M, int H, const double* __restrict__ s,
                                     const double* __restrict__ sums, double dxprod,
                                     double* __restrict__ f, double* __restrict__ fT) {
  __shared__ double tile[32][33];
  const int64_t m0 = (int64_t)blockIdx.x * 32;
  const int h0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int hh = ty; hh < 32; hh += blockDim.y) {
    const int h = h0 + hh;
    const int64_t m = m0 + tx;
    if (h < H && m < M) {
      const int64_t t = (int64_t)h * M + m;
      const double tot = sums[h] * dxprod;
      double v = tot > 0.0 ? s[t] / tot : s[t];
      v = v > 0.0 ? v : 0.0;
      f[t] = v;
      tile[hh][tx] = v;
    }
  }
  __syncthreads();
  for (int mm = ty; mm < 32; mm += blockDim.y) {
    const int64_t m = m0 + mm;
    const int h = h0 + tx;
    if (h < H && m < M) fT[m * H + h] = tile[tx][mm];
  }
}

constexpr int kLcvGroup = 8;  // bandwidths per LCV pass

struct K0g {
  double k0[kLcvGroup];
};

// LCV terms l = log(max(n/(n-1) (f(x_i) - K0/n), 1e-10)) of a group of up to
// kLcvGroup bandwidths h0.. from the bandwidth-fastest densities fT (M, H):
// the trilinear stencil of a point is formed once and each corner's
// densities of the group are contiguous.  Sums of (l - c) and (l - c)^2
// with c = l at point 0: the shift keeps the variance free of cancellation
// (exactly zero when every l is clamped).
template <int D>
__global__ void kde_lcv_group_kernel(InterpGeom g, int64_t n, const double* __restrict__ x,
                                     const double* __restrict__ fT, int H, int h0, int hn, K0g k0,
                                     double* __restrict__ part) {
  __shared__ double sh[32];
  __shared__ double s_c[kLcvGroup], s_k0n[kLcvGroup];
  const double ratio = (double)n / (double)(n - 1);
  if (threadIdx.x < kLcvGroup) {
    const int j = threadIdx.x;
    const double k0n = j < hn ? k0.k0[j] / (double)n : 0.0;
    s_k0n[j] = k0n;
    double c = 0.0;
    if (j < hn) {
      StencilD<D> st;
      make_stencil_d<D>(g, x, 0, st);
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < (1 << D); ++k) v += st.w[k] * fT[st.base[k] * H + h0 + j];
      double fl = ratio * (v - k0n);
      if (!(fl > 1e-10)) fl = 1e-10;
      c = log(fl);
    }
    s_c[j] = c;
  }
  __syncthreads();
  double s1[kLcvGroup], s2[kLcvGroup];
#pragma unroll
  for (int j = 0; j < kLcvGroup; ++j) s1[j] = s2[j] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    StencilD<D> st;
    make_stencil_d<D>(g, x, i, st);
    double v[kLcvGroup];
#pragma unroll
    for (int j = 0; j < kLcvGroup; ++j) v[j] = 0.0;
#pragma unroll
    for (int k = 0; k < (1 << D); ++k) {
      const double* row = fT + st.base[k] * H + h0;
      const double w = st.w[k];
#pragma unroll
      for (int j = 0; j < kLcvGroup; ++j)
        if (j < hn) v[j] += w * row[j];
    }
#pragma unroll
    for (int j = 0; j < kLcvGroup; ++j) {
      if (j < hn) {
        double fl = ratio * (v[j] - s_k0n[j]);
        if (!(fl > 1e-10)) fl = 1e-10;
        const double l = log(fl) - s_c[j];
        s1[j] += l;
        s2[j] += l * l;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kLcvGroup; ++j) {
    if (j < hn) {  // hn is the same for the whole block
      const double a = block_sum(s1[j], sh);
      if (threadIdx.x == 0) atomicAdd(&part[3 * (h0 + j)], a);
      const double b = block_sum(s2[j], sh);
      if (threadIdx.x == 0) {
        atomicAdd(&part[3 * (h0 + j) + 1], b);
        if (blockIdx.x == 0) part[3 * (h0 + j) + 2] = s_c[j];
      }
    }
  }
}

// lcv[h] = {sum l, sum (l - mean)^2} from the shifted sums
__global__ void kde_lcv_finish_kernel(int H, int64_t n, const double* __restrict__ part,
                                      double* __restrict__ lcv) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= H) return;
  const double s1 = part[3 * h], s2 = part[3 * h + 1], c = part[3 * h + 2];
  lcv[2 * h] = (double)n * c + s1;
  const double m2 = s2 - s1 * s1 / (double)n;
  lcv[2 * h + 1] = m2 > 0.0 ? m2 : 0.0;
}

// ---- adjoint of the interpolation (dual form of the GCV/Hutchinson sums) --
// p . interp(m) = sum_g m(g) Q(g) with Q = sum_i w_ig p_i, and
// sum_i interp(m)_i^2 = sum_b sum_{corner pairs} B_b,pair m(b+c) m(b+c'),
// so the point-wise interpolation of every (bandwidth, channel) reduces to
// grid-domain dot products with h-independent deposits Q and B.
__host__ __device__ constexpr int corner_pairs(int d) { return (1 << d) * ((1 << d) + 1) / 2; }

__global__ void deposit_kernel(InterpGeom g, int64_t n, const double* __restrict__ x, int C,
                               ColPtrs vals, double* __restrict__ Q, double* __restrict__ B,
                               double* __restrict__ sq) {
  __shared__ double sh[32];
  const int npair = corner_pairs(g.d);
  double s2[kMaxRed];
#pragma unroll
  for (int c = 0; c < kMaxRed; ++c) s2[c] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    Stencil st;
    make_stencil(g, x, i, st);
#pragma unroll
    for (int c = 0; c < kMaxRed; ++c) {
      if (c < C) {
        const double v = vals.col[c][i];
        s2[c] += v * v;
        for (int k = 0; k < st.ncorner; ++k) atomicAdd(&Q[st.base[k] * C + c], st.w[k] * v);
      }
    }
    int p = 0;
    double* Bb = B + st.base[0] * npair;
    for (int k = 0; k < st.ncorner; ++k)
      for (int k2 = k; k2 < st.ncorner; ++k2, ++p)
        atomicAdd(&Bb[p], (k == k2 ? 1.0 : 2.0) * st.w[k] * st.w[k2]);
  }
#pragma unroll
  for (int c = 0; c < kMaxRed; ++c) {
    if (c < C) {
      double s = block_sum(s2[c], sh);
      if (threadIdx.x == 0) atomicAdd(&sq[c], s);
    }
  }
}

// quad[h][c] = sum_b sum_pairs B[b][pair] m(b+c_k) m(b+c_k2); m: (H, M, ny).
// D fixed at compile time: the 2^D corners and their pairs live in registers.
// blockIdx.y = a chunk of QB bandwidths: each base cell's pair weights are
// read once per chunk and applied to every bandwidth of it.
template <int D>
struct QuadChunk {
  static constexpr int value = D == 3 ? 4 : 8;
};

// part == nullptr: block sums added into quad (atomics); otherwise each
// block's sums go to part[(h * ny + c) * gridDim.x + blockIdx.x] for a
// fixed-order reduction (quad_reduce_kernel): bitwise reproducible
template <int D>
__global__ void stencil_quad_kernel(InterpGeom g, int H, int ny, const double* __restrict__ m,
                                    const double* __restrict__ B, double* __restrict__ quad,
                                    double* __restrict__ part) {
  constexpr int NC = 1 << D;
  constexpr int NP = NC * (NC + 1) / 2;
  constexpr int QB = QuadChunk<D>::value;
  __shared__ double sh[32];
  const int h0 = blockIdx.y * QB;
  int coff[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    int o = 0;
#pragma unroll
    for (int a = 0; a < D; ++a) o = o * g.G[a] + ((k >> (D - 1 - a)) & 1);
    coff[k] = o;
  }
  double acc[QB][4];
#pragma unroll
  for (int q = 0; q < QB; ++q)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[q][c] = 0.0;
  const int M = (int)g.M;  // grids here hold fewer than 2^31 cells
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < M; b += gridDim.x * blockDim.x) {
    // only base cells with every corner inside the grid carry weight
    bool inside = true;
    int r = b;
#pragma unroll
    for (int a = D - 1; a >= 0; --a) {
      const int ia = r % g.G[a];
      r /= g.G[a];
      inside = inside && ia < g.G[a] - 1;
    }
    if (!inside) continue;
    double Bv[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) Bv[p] = B[(int64_t)b * NP + p];
#pragma unroll
    for (int q = 0; q < QB; ++q) {
      if (h0 + q >= H) break;
      const double* mh = m + (int64_t)(h0 + q) * g.M * ny;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= ny) break;
        double mv[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) mv[k] = mh[(int64_t)(b + coff[k]) * ny + c];
        double s = 0.0;
        int p = 0;
#pragma unroll
        for (int k = 0; k < NC; ++k)
#pragma unroll
          for (int k2 = k; k2 < NC; ++k2, ++p) s += Bv[p] * mv[k] * mv[k2];
        acc[q][c] += s;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < QB; ++q) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (h0 + q < H && c < ny) {
        const double s = block_sum(acc[q][c], sh);
        if (threadIdx.x == 0) {
          if (part != nullptr)
            part[((int64_t)(h0 + q) * ny + c) * gridDim.x + blockIdx.x] = s;
          else
            atomicAdd(&quad[(h0 + q) * ny + c], s);
        }
      }
    }
  }
}

// quad[k] = sum of the nb block partials of entry k, in block order
__global__ void quad_reduce_kernel(int nk, int nb, const double* __restrict__ part,
                                   double* __restrict__ quad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[(int64_t)k * nb + b];
  quad[k] = s;
}

static int make_geom(InterpGeom& g, int d, const double* ax, const int* G) {
  memset(&g, 0, sizeof(g));
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "interp: d=%d", d);
  g.d = d;
  g.M = 1;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(G[a] >= 1, "interp: G[%d]=%d", a, G[a]);
    g.G[a] = G[a];
    g.x0[a] = ax[2 * a];
    g.dx[a] = ax[2 * a + 1];
    g.M *= G[a];
  }
  return FLPR_OK;
}

static int pt_blocks(int64_t n, int per_sm) {
  int64_t b = (n + 255) / 256;
  int64_t cap = (int64_t)per_sm * sm_count();
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace flpr

using namespace flpr;

extern "C" {

size_t flpr_interp_reduce_ws(int64_t n, int H, int ny, int R) {
  (void)n;
  (void)H;
  (void)ny;
  (void)R;
  return 0;
}

int flpr_interp_reduce(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G,
                       int H, int ny, int R, const double* d_m, const double* const* h_ycols,
                       const double* const* h_pcols, double* d_rss, double* d_pdot, double* d_pp,
                       void* d_ws, size_t ws_bytes, void* stream) {
  (void)d_ws;
  (void)ws_bytes;
  InterpGeom g;
  FLPR_TRY(make_geom(g, d, h_ax, h_G));
  FLPR_CHECK_ARG(n >= 1 && H >= 1 && ny >= 0 && R >= 0 && ny + R >= 1 && ny + R <= kMaxRed,
                 "interp_reduce: n=%lld H=%d ny=%d R=%d", (long long)n, H, ny, R);
  cudaStream_t s = as_stream(stream);
  ColPtrs yc, pc;
  memset(&yc, 0, sizeof(yc));
  memset(&pc, 0, sizeof(pc));
  for (int c = 0; c < ny; ++c) yc.col[c] = h_ycols[c];
  for (int r = 0; r < R; ++r) pc.col[r] = h_pcols[r];
  if (ny) FLPR_CUDA(cudaMemsetAsync(d_rss, 0, sizeof(double) * H * ny, s));
  if (R) {
    FLPR_CUDA(cudaMemsetAsync(d_pdot, 0, sizeof(double) * H * R, s));
    FLPR_CUDA(cudaMemsetAsync(d_pp, 0, sizeof(double) * R, s));
  }
  int per_h = pt_blocks(n, 4);
  per_h = (per_h + H - 1) / H * 1;
  if (per_h < 8) per_h = 8;
  dim3 grid(per_h, H);
  interp_reduce_kernel<<<grid, 256, 0, s>>>(g, n, d_x, H, ny, R, d_m, yc, pc, d_rss, d_pdot);
  FLPR_LAUNCH_CHECK();
  if (R) {
    probe_norm_kernel<<<pt_blocks(n, 4), 256, 0, s>>>(n, R, pc, d_pp);
    FLPR_LAUNCH_CHECK();
  }
  return FLPR_OK;
}

int flpr_interp_eval(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G,
                     int nval, const double* d_vals, double* d_out, void* stream) {
  InterpGeom g;
  FLPR_TRY(make_geom(g, d, h_ax, h_G));
  FLPR_CHECK_ARG(n >= 1 && nval >= 1, "interp_eval: n=%lld nval=%d", (long long)n, nval);
  interp_eval_kernel<false><<<pt_blocks(n, 8), 256, 0, as_stream(stream)>>>(g, n, d_x, nval,
                                                                             d_vals, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_interp_eval_extrap(int d, int64_t n, const double* d_x, const double* h_ax,
                            const int* h_G, int nval, const double* d_vals, double* d_out,
                            void* stream) {
  InterpGeom g;
  FLPR_TRY(make_geom(g, d, h_ax, h_G));
  FLPR_CHECK_ARG(n >= 1 && nval >= 1, "interp_eval_extrap: n=%lld nval=%d", (long long)n, nval);
  interp_eval_kernel<true><<<pt_blocks(n, 8), 256, 0, as_stream(stream)>>>(g, n, d_x, nval,
                                                                            d_vals, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_deposit(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G, int C,
                 const double* const* h_cols, double* d_Q, double* d_B, double* d_sq,
                 void* stream) {
  InterpGeom g;
  FLPR_TRY(make_geom(g, d, h_ax, h_G));
  FLPR_CHECK_ARG(n >= 1 && C >= 1 && C <= kMaxRed, "deposit: n=%lld C=%d", (long long)n, C);
  for (int a = 0; a < d; ++a) FLPR_CHECK_ARG(h_G[a] >= 2, "deposit: G[%d]=%d < 2", a, h_G[a]);
  cudaStream_t s = as_stream(stream);
  ColPtrs vc;
  memset(&vc, 0, sizeof(vc));
  for (int c = 0; c < C; ++c) vc.col[c] = h_cols[c];
  FLPR_CUDA(cudaMemsetAsync(d_Q, 0, sizeof(double) * (size_t)g.M * C, s));
  FLPR_CUDA(cudaMemsetAsync(d_B, 0, sizeof(double) * (size_t)g.M * corner_pairs(d), s));
  FLPR_CUDA(cudaMemsetAsync(d_sq, 0, sizeof(double) * C, s));
  deposit_kernel<<<pt_blocks(n, 8), 256, 0, s>>>(g, n, d_x, C, vc, d_Q, d_B, d_sq);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

static int quad_grid(const InterpGeom& g, int H, int* per, int* nchunk) {
  const int qb = g.d == 3 ? QuadChunk<3>::value : QuadChunk<2>::value;
  *nchunk = (H + qb - 1) / qb;
  int p = (pt_blocks(g.M, 4) + *nchunk - 1) / *nchunk;
  if (p < 4) p = 4;
  *per = p;
  return FLPR_OK;
}

static int stencil_quad_impl(int d, const int* h_G, int H, int ny, const double* d_m,
                             const double* d_B, double* d_quad, double* d_part, void* stream) {
  InterpGeom g;
  double ax[6] = {0, 1, 0, 1, 0, 1};
  FLPR_TRY(make_geom(g, d, ax, h_G));
  FLPR_CHECK_ARG(H >= 1 && ny >= 1 && ny <= 4, "stencil_quad: H=%d ny=%d", H, ny);
  cudaStream_t s = as_stream(stream);
  FLPR_CHECK_ARG(g.M < ((int64_t)1 << 31), "stencil_quad: grid too large");
  int per, nchunk;
  quad_grid(g, H, &per, &nchunk);
  if (d_part == nullptr) FLPR_CUDA(cudaMemsetAsync(d_quad, 0, sizeof(double) * H * ny, s));
  switch (d) {
    case 1: stencil_quad_kernel<1><<<dim3(per, nchunk), 256, 0, s>>>(g, H, ny, d_m, d_B, d_quad, d_part); break;
    case 2: stencil_quad_kernel<2><<<dim3(per, nchunk), 256, 0, s>>>(g, H, ny, d_m, d_B, d_quad, d_part); break;
    default: stencil_quad_kernel<3><<<dim3(per, nchunk), 256, 0, s>>>(g, H, ny, d_m, d_B, d_quad, d_part); break;
  }
  FLPR_LAUNCH_CHECK();
  if (d_part != nullptr) {
    const int nk = H * ny;
    quad_reduce_kernel<<<(nk + 127) / 128, 128, 0, s>>>(nk, per, d_part, d_quad);
    FLPR_LAUNCH_CHECK();
  }
  return FLPR_OK;
}

int flpr_stencil_quad(int d, const int* h_G, int H, int ny, const double* d_m, const double* d_B,
                      double* d_quad, void* stream) {
  return stencil_quad_impl(d, h_G, H, ny, d_m, d_B, d_quad, nullptr, stream);
}

size_t flpr_stencil_quad_fixed_ws(int d, const int* h_G, int H, int ny) {
  InterpGeom g;
  double ax[6] = {0, 1, 0, 1, 0, 1};
  if (make_geom(g, d, ax, h_G) != FLPR_OK || H < 1 || ny < 1) return 0;
  int per, nchunk;
  quad_grid(g, H, &per, &nchunk);
  return align_up(sizeof(double) * (size_t)per * (size_t)H * (size_t)ny);
}

int flpr_stencil_quad_fixed(int d, const int* h_G, int H, int ny, const double* d_m,
                            const double* d_B, double* d_quad, void* d_ws, size_t ws_bytes,
                            void* stream) {
  FLPR_CHECK_ARG(d_ws != nullptr, "stencil_quad_fixed: null workspace");
  if (ws_bytes < flpr_stencil_quad_fixed_ws(d, h_G, H, ny)) {
    set_error("stencil_quad_fixed: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  return stencil_quad_impl(d, h_G, H, ny, d_m, d_B, d_quad, static_cast<double*>(d_ws), stream);
}

size_t flpr_kde_ws(int64_t n, int H, int64_t M) {
  (void)n;
  const size_t h = (size_t)(H > 0 ? H : 1);
  return align_up(sizeof(double) * h) + align_up(sizeof(double) * 3 * h) +
         align_up(sizeof(double) * h * (size_t)(M > 0 ? M : 1));
}

int flpr_kde_lcv(int d, int64_t n, const double* d_x, const double* h_ax, const int* h_G, int H,
                 const double* d_s, double dxprod, const double* h_k0, double* d_f, double* d_lcv,
                 void* d_ws, size_t ws_bytes, void* stream) {
  InterpGeom g;
  FLPR_TRY(make_geom(g, d, h_ax, h_G));
  FLPR_CHECK_ARG(n >= 2 && H >= 1, "kde_lcv: n=%lld H=%d", (long long)n, H);
  if (ws_bytes < flpr_kde_ws(n, H, g.M)) {
    set_error("kde_lcv: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  cudaStream_t s = as_stream(stream);
  double* sums = static_cast<double*>(d_ws);
  double* part = reinterpret_cast<double*>(static_cast<char*>(d_ws) +
                                           align_up(sizeof(double) * (size_t)H));
  FLPR_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * H, s));
  FLPR_CUDA(cudaMemsetAsync(part, 0, sizeof(double) * 3 * H, s));
  int gb = pt_blocks(g.M, 2);
  gb = (gb + H - 1) / H;
  if (gb < 4) gb = 4;
  plane_sum_kernel<<<dim3(gb, H), 256, 0, s>>>(g.M, d_s, sums);
  FLPR_LAUNCH_CHECK();
  double* fT = reinterpret_cast<double*>(static_cast<char*>(d_ws) +
                                         align_up(sizeof(double) * (size_t)H) +
                                         align_up(sizeof(double) * 3 * (size_t)H));
  FLPR_CHECK_ARG((g.M + 31) / 32 < ((int64_t)1 << 31), "kde_lcv: grid too large");
  kde_normalize_kernel<<<dim3((unsigned)((g.M + 31) / 32), (unsigned)((H + 31) / 32)),
                         dim3(32, 8), 0, s>>>(g.M, H, d_s, sums, dxprod, d_f, fT);
  FLPR_LAUNCH_CHECK();
  const int ngroups = (H + kLcvGroup - 1) / kLcvGroup;
  const int per_g = (4 * sm_count() + ngroups - 1) / ngroups;
  for (int h0 = 0; h0 < H; h0 += kLcvGroup) {
    const int hn = H - h0 < kLcvGroup ? H - h0 : kLcvGroup;
    K0g k0;
    for (int j = 0; j < kLcvGroup; ++j) k0.k0[j] = j < hn ? h_k0[h0 + j] : 0.0;
    switch (d) {
      case 1: kde_lcv_group_kernel<1><<<per_g, 256, 0, s>>>(g, n, d_x, fT, H, h0, hn, k0, part); break;
      case 2: kde_lcv_group_kernel<2><<<per_g, 256, 0, s>>>(g, n, d_x, fT, H, h0, hn, k0, part); break;
      default: kde_lcv_group_kernel<3><<<per_g, 256, 0, s>>>(g, n, d_x, fT, H, h0, hn, k0, part); break;
    }
    FLPR_LAUNCH_CHECK();
  }
  kde_lcv_finish_kernel<<<(H + 127) / 128, 128, 0, s>>>(H, n, part, d_lcv);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
