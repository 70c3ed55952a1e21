// Direct separable 2-D convolution for short kernel stencils.
//
// The FFT convolution of a grid with the per-axis kernel factor arrays
// (flpr_kernel_factors samples v(k) = exp(-u^2/2) u^p / h, u = g_k / h, at
// the kernel-grid nodes g_k and places node k at index k + (L - G)/2 + 1 of
// an L-array) is the circular convolution
//   out(x) = scale * L0 * L1 * sum_{i0, i1} arr0(i0) arr1(i1) grid(x - i)
// cropped to x in [qout, qout + G).  For a bandwidth of a few grid cells the
// arrays are negligible (below 1e-22 of their peak: |u| > 11) outside a few
// dozen nodes, so the sum over those nodes replaces two transforms per
// product: the FP64 planes of the bandwidths whose kernel covers few points
// (the FP64 group of the FP32 path) cost a small fraction of their
// transforms.  Three launches: the stencils (the factor samples, in the
// same operation order as the factor arrays), the axis-0 pass per (channel,
// axis-0 power, bandwidth) over every column, and the axis-1 pass per
// product into the cropped planes.  The index tables travel as kernel
// arguments, so a call needs no host round trip (and can be captured).
#include "common.cuh"

namespace flpr {
namespace {

constexpr int kDirMaxTaps = 160;     // stencil nodes per axis
constexpr int kDirMaxH = 32;         // bandwidths per call
constexpr int kDirMaxItems = 128;    // slots and products per call
constexpr double kDirTail = 11.0;    // |u| beyond which the factors are below 1e-22

struct DirArgs {
  int G[2], L[2], q[2], before[2];
  double lo[2], hi[2], step[2];
  int H, npow;
  short k0[2][kDirMaxH];   // first stencil node per (axis, bandwidth)
  short nk[2][kDirMaxH];   // stencil nodes per (axis, bandwidth)
  double h[2][kDirMaxH];   // bandwidth per (axis, bandwidth)
};

struct DirTables {
  int nslots, nprod;
  short slot_c[kDirMaxItems], slot_a0[kDirMaxItems], slot_h[kDirMaxItems];
  short prod_slot[kDirMaxItems], prod_a1[kDirMaxItems];
  int prod_out[kDirMaxItems];   // plane index of each product in the output
};

// st[((a * H + h) * npow + p) * kDirMaxTaps + t] = v(k0 + t), in the
// operation order of the kernel factor samples (no contraction)
__global__ void stencil_kernel(DirArgs da, double* __restrict__ st) {
  const int row = blockIdx.x;  // (a, h, p)
  const int a = row / (da.H * da.npow);
  const int r = row - a * da.H * da.npow;
  const int hi_ = r / da.npow, p = r - hi_ * da.npow;
  const double hv = da.h[a][hi_];
  const int G = da.G[a];
  for (int t = threadIdx.x; t < kDirMaxTaps; t += blockDim.x) {
    double v = 0.0;
    if (t < da.nk[a][hi_]) {
      const int k = da.k0[a][hi_] + t;
      const double g = (k == G - 1 && G > 1) ? da.hi[a]
                                              : __dadd_rn(__dmul_rn((double)k, da.step[a]), da.lo[a]);
      const double u = __ddiv_rn(g, hv);
      const double e = exp(__dmul_rn(-0.5, __dmul_rn(u, u)));
      double pw = 1.0;
      for (int q = 0; q < p; ++q) pw = __dmul_rn(pw, u);
      v = __ddiv_rn(__dmul_rn(e, pw), hv);
    }
    st[(size_t)row * kDirMaxTaps + t] = v;
  }
}

// Axis-0 pass: tmp[slot][x0][w1] = sum_t st0(h, a0, t) grid[c][(x0 + q0 - i0) mod L0][w1],
// i0 = k0 + t + before0; grid (ceil(L1 / 128), G0, nslots), 128 threads.
__global__ void dir_pass0_kernel(DirArgs da, DirTables tb, const double* __restrict__ grid,
                                 const double* __restrict__ st, double* __restrict__ tmp) {
  const int w1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int x0 = blockIdx.y, sl = blockIdx.z;
  if (w1 >= da.L[1] || sl >= tb.nslots) return;
  const int c = tb.slot_c[sl], a0 = tb.slot_a0[sl], h = tb.slot_h[sl];
  const int L0 = da.L[0], L1 = da.L[1];
  const double* s = st + ((size_t)h * da.npow + a0) * kDirMaxTaps;
  const double* gc = grid + (size_t)c * L0 * L1 + w1;
  const int base = x0 + da.q[0] - da.k0[0][h] - da.before[0];
  const int nk = da.nk[0][h];
  double acc = 0.0;
  for (int t = 0; t < nk; ++t) {
    int r = (base - t) % L0;
    if (r < 0) r += L0;
    acc = fma(s[t], gc[(size_t)r * L1], acc);
  }
  tmp[((size_t)sl * da.G[0] + x0) * L1 + w1] = acc;
}

// Axis-1 pass: out[p][x0 * G1 + x1] = f * sum_t st1(h, a1, t) tmp[slot][x0][(x1 + q1 - i1) mod L1];
// grid (ceil(G1 / 128), G0, nprod), 128 threads.
__global__ void dir_pass1_kernel(DirArgs da, DirTables tb, const double* __restrict__ st,
                                 const double* __restrict__ tmp, double f, int add_eps,
                                 double* __restrict__ out) {
  const int x1 = blockIdx.x * blockDim.x + threadIdx.x;
  const int x0 = blockIdx.y, pr = blockIdx.z;
  if (x1 >= da.G[1] || pr >= tb.nprod) return;
  const int sl = tb.prod_slot[pr], a1 = tb.prod_a1[pr], h = tb.slot_h[sl];
  const int L1 = da.L[1];
  const double* s = st + ((size_t)(da.H + h) * da.npow + a1) * kDirMaxTaps;
  const double* row = tmp + ((size_t)sl * da.G[0] + x0) * L1;
  const int base = x1 + da.q[1] - da.k0[1][h] - da.before[1];
  const int nk = da.nk[1][h];
  double acc = 0.0;
  for (int t = 0; t < nk; ++t) {
    int r = (base - t) % L1;
    if (r < 0) r += L1;
    acc = fma(s[t], row[r], acc);
  }
  double v = f * acc;
  if (add_eps) v += 2.220446049250313e-16;
  out[(size_t)tb.prod_out[pr] * da.G[0] * da.G[1] + (size_t)x0 * da.G[1] + x1] = v;
}

// Stencil node range of one (axis, bandwidth): the nodes with |g / h| <= 11.
static void node_range(int G, double lo, double hi, double h, int* k0, int* nk) {
  const double step = G > 1 ? (hi - lo) / (double)(G - 1) : 0.0;
  if (!(step > 0.0) || !(h > 0.0)) {
    *k0 = 0;
    *nk = G;
    return;
  }
  int a = (int)floor((-kDirTail * h - lo) / step) - 1;
  int b = (int)ceil((kDirTail * h - lo) / step) + 1;
  if (a < 0) a = 0;
  if (b > G - 1) b = G - 1;
  *k0 = a;
  *nk = b >= a ? b - a + 1 : 0;
}

static int dir_args(const int* G, const int* L, const int* q, const double* lo, const double* hi,
                    int H, int npow, const double* h_bw, DirArgs* da) {
  memset(da, 0, sizeof(*da));
  if (H < 1 || H > kDirMaxH) {
    set_error("conv2d_direct: H=%d not in [1, %d]", H, kDirMaxH);
    return FLPR_ERR_ARG;
  }
  if (npow < 1 || npow > 5) {
    set_error("conv2d_direct: npow=%d", npow);
    return FLPR_ERR_ARG;
  }
  da->H = H;
  da->npow = npow;
  for (int a = 0; a < 2; ++a) {
    if (!(G[a] >= 2 && L[a] >= G[a] && q[a] >= 0 && q[a] + G[a] <= L[a])) {
      set_error("conv2d_direct: grid/crop axis %d", a);
      return FLPR_ERR_ARG;
    }
    da->G[a] = G[a];
    da->L[a] = L[a];
    da->q[a] = q[a];
    da->before[a] = (L[a] - G[a]) / 2 + 1;
    da->lo[a] = lo[a];
    da->hi[a] = hi[a];
    da->step[a] = (hi[a] - lo[a]) / (double)(G[a] - 1);
    for (int h = 0; h < H; ++h) {
      int k0 = 0, nk = 0;
      node_range(G[a], lo[a], hi[a], h_bw[h * 2 + a], &k0, &nk);
      if (nk > kDirMaxTaps) {
        set_error("conv2d_direct: stencil of %d nodes (max %d)", nk, kDirMaxTaps);
        return FLPR_ERR_ARG;
      }
      da->h[a][h] = h_bw[h * 2 + a];
      da->k0[a][h] = (short)k0;
      da->nk[a][h] = (short)nk;
    }
  }
  return FLPR_OK;
}

}  // namespace
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_conv2d_direct_supported(const int* h_G, const int* h_L, const int* h_qout,
                                 const double* h_lo, const double* h_hi, int H, int npow,
                                 const double* h_bw) {
  DirArgs da;
  return dir_args(h_G, h_L, h_qout, h_lo, h_hi, H, npow, h_bw, &da) == FLPR_OK ? 1 : 0;
}

size_t flpr_conv2d_direct_ws(const int* h_G, const int* h_L, int H, int npow, int nslots) {
  if (H < 1 || nslots < 1 || !h_G || !h_L) return 0;
  ArenaSize ar;
  ar.take<double>((size_t)2 * H * npow * kDirMaxTaps);
  ar.take<double>((size_t)nslots * h_G[0] * h_L[1]);
  return ar.used;
}

int flpr_conv2d_direct(const int* h_G, const int* h_L, const int* h_qout, const double* h_lo,
                       const double* h_hi, int H, int npow, const double* h_bw, double scale,
                       const double* d_grid, int nprod, const int* h_chan, const int* h_hidx,
                       const int* h_pow, const int* h_out_index, int add_eps, double* d_out,
                       void* d_ws, size_t ws_bytes, void* stream) {
  DirArgs da;
  FLPR_TRY(dir_args(h_G, h_L, h_qout, h_lo, h_hi, H, npow, h_bw, &da));
  FLPR_CHECK_ARG(nprod >= 1 && nprod <= kDirMaxItems && d_grid && d_out,
                 "conv2d_direct: %d products (max %d) / pointers", nprod, kDirMaxItems);
  // slots: distinct (channel, axis-0 power, bandwidth) of the products
  DirTables tb;
  memset(&tb, 0, sizeof(tb));
  for (int p = 0; p < nprod; ++p) {
    const int c = h_chan[p], h = h_hidx[p], a0 = h_pow[2 * p], a1 = h_pow[2 * p + 1];
    FLPR_CHECK_ARG(h >= 0 && h < H && a0 >= 0 && a0 < npow && a1 >= 0 && a1 < npow && c >= 0 &&
                       c < 32768,
                   "conv2d_direct: product %d", p);
    int found = -1;
    for (int s = 0; s < tb.nslots; ++s)
      if (tb.slot_c[s] == c && tb.slot_a0[s] == a0 && tb.slot_h[s] == h) found = s;
    if (found < 0) {
      found = tb.nslots++;
      tb.slot_c[found] = (short)c;
      tb.slot_a0[found] = (short)a0;
      tb.slot_h[found] = (short)h;
    }
    tb.prod_slot[p] = (short)found;
    tb.prod_a1[p] = (short)a1;
    tb.prod_out[p] = h_out_index ? h_out_index[p] : p;
    FLPR_CHECK_ARG(tb.prod_out[p] >= 0, "conv2d_direct: output index of product %d", p);
  }
  tb.nprod = nprod;
  const size_t need = flpr_conv2d_direct_ws(h_G, h_L, H, npow, tb.nslots);
  if (ws_bytes < need) {
    set_error("conv2d_direct: workspace too small (%zu < %zu)", ws_bytes, need);
    return FLPR_ERR_WORKSPACE;
  }
  Arena ar(d_ws, ws_bytes);
  double* st = ar.take<double>((size_t)2 * H * npow * kDirMaxTaps);
  double* tmp = ar.take<double>((size_t)tb.nslots * h_G[0] * h_L[1]);
  cudaStream_t s = as_stream(stream);
  stencil_kernel<<<2 * H * npow, 128, 0, s>>>(da, st);
  FLPR_LAUNCH_CHECK();
  dir_pass0_kernel<<<dim3((h_L[1] + 127) / 128, h_G[0], tb.nslots), 128, 0, s>>>(da, tb, d_grid,
                                                                               st, tmp);
  FLPR_LAUNCH_CHECK();
  const double f = scale * (double)h_L[0] * (double)h_L[1];
  dir_pass1_kernel<<<dim3((h_G[1] + 127) / 128, h_G[0], nprod), 128, 0, s>>>(da, tb, st, tmp, f,
                                                                           add_eps, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
