// Gaussian-gridding spread (NUFFT type-1 spreading) of many channels.
//
// Pipeline (all on one stream):
//   1. bin_count   : knot mapping per point, home cell -> tile id, tile
//                    histogram; per-channel sum |v| (sets the fixed-point
//                    scale of the FP32 path).
//   2. tile_scan   : exclusive scans of the histogram and of the number of
//                    work items per tile (a tile is split into chunks of at
//                    most FLPR_TUNE_SPREAD_ITEM_POINTS points).
//   3. bin_scatter : point indices sorted by tile.
//   4. tile_accumulate : one CTA per work item; every point of the chunk is
//                    spread into a shared-memory copy of its tile plus a
//                    halo of msp cells (one warp per point, lanes over taps),
//                    then the tile is added to the global accumulator with
//                    one atomic per non-zero cell.
//   5. finalize    : accumulator -> real grid (float or double) times 1/n.
//
// FLPR_PREC_F32 accumulates 64-bit fixed point: integer addition is
// associative, so the result does not depend on the order of the atomics
// and the grid is deterministic.  FLPR_PREC_F64 accumulates float64.
#include "common.cuh"

namespace flpr {

// points per work item: tuning(FLPR_TUNE_SPREAD_ITEM_POINTS), carried in SpreadGeom
constexpr int kSpreadThreads = 256;
constexpr int kMaxTaps1 = 25;  // 2*msp+1 for msp <= 12 (msp = 0: binning with weight 1)

struct SpreadGeom {
  int d;
  int L[3];
  int T[3];        // tile extent per axis
  int ntile[3];    // tiles per axis
  int W[3];        // tile + halo extent per axis
  int msp;
  int ntaps1;      // 2*msp+1
  int64_t cells;   // prod(L)
  int tile_cells;  // prod(W)
  int ntiles;
  int item_points;  // points per work item (one CTA)
  double four_tau[3];
  KnotAxis ax[3];
};

struct ChanPtrs {
  const double* col[FLPR_MAX_CHANNELS];
};

// Home cell and tile of a point; also its unwrapped knot index m.  ax: the
// knot maps of the axes (the geometry's, or a device-computed copy).
__device__ __forceinline__ int point_tile(const SpreadGeom& g, const KnotAxis* ax,
                                          const double* __restrict__ x, int64_t i, int* m_out,
                                          double* k_out) {
  int tile = 0;
  for (int a = 0; a < g.d; ++a) {
    double k = knot_of(x[i * g.d + a], ax[a]);
    int m = (int)rint(ddiv(k, ax[a].hx));
    int home = m % g.L[a];
    if (home < 0) home += g.L[a];
    tile = tile * g.ntile[a] + home / g.T[a];
    if (m_out) m_out[a] = m;
    if (k_out) k_out[a] = k;
  }
  return tile;
}

// Knot maps of the axes into shared memory: from d_kmap (d x 9, the layout
// of the host geometry's rows) when given, else from the geometry.
__device__ __forceinline__ void load_axes(const SpreadGeom& g, const double* __restrict__ d_kmap,
                                          KnotAxis* s_ax) {
  if (threadIdx.x < g.d) {
    const int a = threadIdx.x;
    if (d_kmap) {
      const double* k = d_kmap + 9 * a;
      s_ax[a] = KnotAxis{k[0], k[1], k[2], k[3], k[4], k[5], k[6], k[7], k[8]};
    } else {
      s_ax[a] = g.ax[a];
    }
  }
}

// Knot maps (d x 9: mean, std, centre, centred minimum, scale, ks, r0, shift,
// hx) from the point statistics (4 x d: minimum, maximum, mean, M2), with
// the operations, in the order, of the host geometry: z-score with ddof 1
// (model.py:58-68), mid-range centring, the knot-range mapping
// (convolution.py:190-208) and the centring shift (nufftn_type1.py:164-166).
// One thread per axis.  nm1 = n - 1 (negative for one point: std NaN).
struct KnotConsts {
  double ks[3], r0[3], hx[3];
};

__global__ void knot_map_kernel(int d, double nm1, const double* __restrict__ st, KnotConsts kc,
                                double* __restrict__ kmap) {
  const int a = threadIdx.x;
  if (a >= d) return;
  const double xmin = st[a], xmax = st[d + a], mean = st[2 * d + a], m2 = st[3 * d + a];
  double sd = nm1 > 0.0 ? __dsqrt_rn(ddiv(m2, nm1)) : NAN;
  if (sd == 0.0) sd = 1.0;
  const double xs_min = ddiv(dsub(xmin, mean), sd);
  const double xs_max = ddiv(dsub(xmax, mean), sd);
  const double center = ddiv(dadd(xs_max, xs_min), 2.0);
  const double lo = dsub(xs_min, center);
  const double hi = dsub(xs_max, center);
  double scale = dsub(hi, lo);
  if (scale == 0.0) scale = 1.0;
  const double ks = kc.ks[a], r0 = kc.r0[a];
  double c[2];
  for (int e = 0; e < 2; ++e) {
    double xn = dadd(dmul(ddiv(dsub(e == 0 ? lo : hi, lo), scale), ks), r0);
    xn = dadd(xn, 0.5);
    xn = np_mod(xn, 1.0);
    c[e] = dsub(xn, 0.5);
  }
  const double kmin = dsub(dmul(dadd(c[0], c[1]), 0.5), 0.5);
  const double shift = dsub(-0.5, kmin);
  double* o = kmap + 9 * a;
  o[0] = mean;
  o[1] = sd;
  o[2] = center;
  o[3] = lo;
  o[4] = scale;
  o[5] = ks;
  o[6] = r0;
  o[7] = shift;
  o[8] = kc.hx[a];
}

__global__ void bin_count_kernel(SpreadGeom g, int64_t n, const double* __restrict__ x,
                                 const double* __restrict__ d_kmap,
                                 int* __restrict__ point_tile_out, int* __restrict__ counts,
                                 int nchan, int ones_channel, ChanPtrs cp,
                                 double* __restrict__ absum) {
  __shared__ double sh_abs[FLPR_MAX_CHANNELS];
  __shared__ KnotAxis s_ax[3];
  for (int c = threadIdx.x; c < nchan; c += blockDim.x) sh_abs[c] = 0.0;
  load_axes(g, d_kmap, s_ax);
  __syncthreads();
  int nv = nchan - ones_channel;
  double local[8];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int t = point_tile(g, s_ax, x, i, nullptr, nullptr);
    point_tile_out[i] = t;
    atomicAdd(&counts[t], 1);
  }
  if (absum != nullptr) {
    // per-channel sum of |v| in chunks of 8 channels per sweep
    for (int c0 = 0; c0 < nv; c0 += 8) {
      int cn = min(8, nv - c0);
      for (int c = 0; c < 8; ++c) local[c] = 0.0;
      for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
           i += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < cn; ++c) local[c] += fabs(cp.col[c0 + c][i]);
      for (int c = 0; c < cn; ++c) {
        double v = local[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sh_abs[ones_channel + c0 + c], v);
      }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nchan; c += blockDim.x) {
      if (ones_channel && c == 0) {
        if (blockIdx.x == 0) atomicAdd(&absum[0], (double)n);
      } else {
        atomicAdd(&absum[c], sh_abs[c]);
      }
    }
  }
}

// Single-block exclusive scans over the tile histogram (points and work
// items per tile): per 1024-tile chunk a warp-shuffle scan, the warp totals
// scanned by warp 0, and a running carry.  Launched with 1024 threads.
__global__ void tile_scan_kernel(int ntiles, int item_points, const int* __restrict__ counts,
                                 int* __restrict__ offsets, int* __restrict__ items,
                                 int* __restrict__ cursor) {
  __shared__ int wa[32], wb[32];
  __shared__ int carry_a, carry_b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    carry_a = 0;
    carry_b = 0;
  }
  __syncthreads();
  for (int base = 0; base < ntiles; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const int c = t < ntiles ? counts[t] : 0;
    const int a = c;
    const int b = (c + item_points - 1) / item_points;
    int ia = a, ib = b;  // inclusive warp scans
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int va = __shfl_up_sync(0xffffffffu, ia, o);
      const int vb = __shfl_up_sync(0xffffffffu, ib, o);
      if (lane >= o) {
        ia += va;
        ib += vb;
      }
    }
    if (lane == 31) {
      wa[warp] = ia;
      wb[warp] = ib;
    }
    __syncthreads();
    if (warp == 0) {
      int xa = wa[lane], xb = wb[lane];  // 32 warps of 32 threads
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int va = __shfl_up_sync(0xffffffffu, xa, o);
        const int vb = __shfl_up_sync(0xffffffffu, xb, o);
        if (lane >= o) {
          xa += va;
          xb += vb;
        }
      }
      wa[lane] = xa;  // inclusive warp totals
      wb[lane] = xb;
    }
    __syncthreads();
    const int pa = carry_a + (warp ? wa[warp - 1] : 0) + ia - a;
    const int pb = carry_b + (warp ? wb[warp - 1] : 0) + ib - b;
    if (t < ntiles) {
      offsets[t] = pa;
      items[t] = pb;
      cursor[t] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      carry_a += wa[31];
      carry_b += wb[31];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    offsets[ntiles] = carry_a;
    items[ntiles] = carry_b;
  }
}

// Sorted structure-of-arrays records, one slot per point in tile order:
//   rec_base[pos]          local base cell of the point inside its tile,
//                          packed 10 bits per axis (T <= 1024);
//   rec_frac[a * n + pos]  k_a - hx_a * m_a (offset of the knot from its cell);
//   rec_val[c * n + pos]   value of channel c (ones channel excluded).
template <typename Real>
__global__ void bin_scatter_kernel(SpreadGeom g, int64_t n, const double* __restrict__ x,
                                   const double* __restrict__ d_kmap,
                                   const int* __restrict__ offsets, int* __restrict__ cursor,
                                   int nv, ChanPtrs cp, int* __restrict__ rec_base,
                                   int* __restrict__ rec_idx, Real* __restrict__ rec_frac,
                                   Real* __restrict__ rec_val) {
  __shared__ KnotAxis s_ax[3];
  load_axes(g, d_kmap, s_ax);
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int m[3];
    double k[3];
    const int t = point_tile(g, s_ax, x, i, m, k);
    const int pos = offsets[t] + atomicAdd(&cursor[t], 1);
    int packed = 0;
    for (int a = 0; a < g.d; ++a) {
      int home = m[a] % g.L[a];
      if (home < 0) home += g.L[a];
      packed |= (home % g.T[a]) << (10 * a);
      rec_frac[(int64_t)a * n + pos] = (Real)dsub(k[a], dmul(g.ax[a].hx, (double)m[a]));
    }
    rec_base[pos] = packed;
    rec_idx[pos] = (int)i;
    for (int c = 0; c < nv; ++c) rec_val[(int64_t)c * n + pos] = (Real)cp.col[c][i];
  }
}

template <typename Acc>
struct AccOps;

template <>
struct AccOps<long long> {
  template <typename Real>
  __device__ static void add_shared(long long* p, Real v, Real scale) {
    long long q = (sizeof(Real) == 4) ? __float2ll_rn((float)(v * scale))
                                      : __double2ll_rn((double)(v * scale));
    if (q != 0) atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)q);
  }
  __device__ static void add_global(long long* p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
  }
};

template <>
struct AccOps<double> {
  template <typename Real>
  __device__ static void add_shared(double* p, Real v, Real) { atomicAdd(p, (double)v); }
  __device__ static void add_global(double* p, double v) { atomicAdd(p, v); }
};

// Fixed-point scale 2^e per channel so that |sum| over any subset of
// contributions stays below 2^50 (each point adds at most |v| to a cell when
// the taps do not wrap onto the same cell): every rounded product and every
// partial sum is then an integer that a double holds exactly, so the 2-D
// path can round and add in FP64 registers and still be exact and
// independent of the order of the points.  The quantum, 2^-50 of the
// channel's absolute sum, is far below the FP32 rounding of the grid.
constexpr int kFixedBits = 50;

__device__ __forceinline__ double fixed_scale(double absum, int margin_bits) {
  if (!(absum > 0.0)) return 1.0;
  int e = 0;
  frexp(absum, &e);  // absum < 2^e
  return ldexp(1.0, kFixedBits - e - margin_bits);
}

__device__ __forceinline__ float fexp(float v) { return expf(v); }
__device__ __forceinline__ double fexp(double v) { return exp(v); }

// One CTA per work item (a tile, or a chunk of at most g.item_points points of
// a tile).  Threads take (point, tap row) pairs: a tap row fixes the tap
// offsets of all axes but the last, and the thread walks the NT1 taps of the
// last axis, adding every channel of the point into the shared-memory copy of
// the tile plus its halo of msp cells.  The tile is then added to the global
// accumulator with one atomic per non-zero cell.
template <typename Acc, typename Real, int NT1>
__global__ void __launch_bounds__(kSpreadThreads)
tile_accumulate_kernel(SpreadGeom g, int64_t n, int nchan, int ones_channel, int cgroup,
                       const int* __restrict__ offsets, const int* __restrict__ items,
                       const int* __restrict__ rec_base, const Real* __restrict__ rec_frac,
                       const Real* __restrict__ rec_val, const double* __restrict__ absum,
                       int margin_bits, Acc* __restrict__ gacc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Acc* acc = reinterpret_cast<Acc*>(smem_raw);
  const int c_begin = blockIdx.y * cgroup;
  const int nc = min(nchan, c_begin + cgroup) - c_begin;
  const int tc = g.tile_cells;

  const int item = blockIdx.x;
  if (item >= items[g.ntiles]) return;
  int lo = 0, hi = g.ntiles;  // tile owning this item: largest t with items[t] <= item
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (items[mid] <= item) lo = mid; else hi = mid;
  }
  const int tile = lo;
  const int p_begin = offsets[tile] + (item - items[tile]) * g.item_points;
  const int p_end = min(offsets[tile + 1], p_begin + g.item_points);
  int tcoord[3] = {0, 0, 0};
  {
    int r = tile;
    for (int a = g.d - 1; a >= 0; --a) {
      tcoord[a] = r % g.ntile[a];
      r /= g.ntile[a];
    }
  }
  __shared__ Real scale[32];
  for (int i = threadIdx.x; i < nc * tc; i += blockDim.x) acc[i] = Acc(0);
  if (threadIdx.x < 32)
    scale[threadIdx.x] = (threadIdx.x < nc)
                             ? (Real)fixed_scale(absum ? absum[c_begin + threadIdx.x] : 0.0, margin_bits)
                             : Real(1);
  __syncthreads();

  constexpr int MSP = (NT1 - 1) / 2;
  const int d = g.d;
  const int rows = d == 1 ? 1 : (d == 2 ? NT1 : NT1 * NT1);
  const int np = p_end - p_begin;
  const int Wl = g.W[d - 1];
  const Real hxl = (Real)g.ax[d - 1].hx;
  const Real ftl = (Real)g.four_tau[d - 1];
  for (int t = threadIdx.x; t < np * rows; t += blockDim.x) {
    const int pp = t / rows;
    const int p = p_begin + pp;
    const int row = t - pp * rows;
    const int packed = rec_base[p];
    int j[2] = {0, 0};
    if (d == 2) {
      j[0] = row;
    } else if (d == 3) {
      j[0] = row / NT1;
      j[1] = row - j[0] * NT1;
    }
    // weight and local cell of the tap row (all axes but the last)
    Real wrow = Real(1);
    int cell = 0;
    for (int a = 0; a < d - 1; ++a) {
      const Real fr = rec_frac[(int64_t)a * n + p];
      const Real diff = fr - (Real)g.ax[a].hx * (Real)(j[a] - MSP);
      wrow *= fexp(-(diff * diff) / (Real)g.four_tau[a]);
      cell = cell * g.W[a] + ((packed >> (10 * a)) & 1023) + j[a];
    }
    cell = cell * Wl + ((packed >> (10 * (d - 1))) & 1023);
    const Real frl = rec_frac[(int64_t)(d - 1) * n + p];
    Real w[NT1];
#pragma unroll
    for (int jl = 0; jl < NT1; ++jl) {
      const Real diff = frl - hxl * (Real)(jl - MSP);
      w[jl] = wrow * fexp(-(diff * diff) / ftl);
    }
    for (int c = 0; c < nc; ++c) {
      const int ch = c_begin + c;
      const Real v = (ones_channel && ch == 0) ? Real(1) : rec_val[(int64_t)(ch - ones_channel) * n + p];
      const Real sc = scale[c];
      Acc* dst = acc + c * tc + cell;
#pragma unroll
      for (int jl = 0; jl < NT1; ++jl) AccOps<Acc>::add_shared(dst + jl, v * w[jl], sc);
    }
  }
  __syncthreads();

  // flush: one global atomic per non-zero cell of the tile + halo
  for (int idx = threadIdx.x; idx < nc * tc; idx += blockDim.x) {
    Acc v = acc[idx];
    if (v == Acc(0)) continue;
    int c = idx / tc;
    int r = idx - c * tc;
    int64_t gi = 0;
    int loc[3] = {0, 0, 0};
    for (int a = g.d - 1; a >= 0; --a) {
      loc[a] = r % g.W[a];
      r /= g.W[a];
    }
    for (int a = 0; a < g.d; ++a) {
      int gc = tcoord[a] * g.T[a] + loc[a] - g.msp;
      gc %= g.L[a];
      if (gc < 0) gc += g.L[a];
      gi = gi * g.L[a] + gc;
    }
    AccOps<Acc>::add_global(&gacc[(int64_t)(c_begin + c) * g.cells + gi], v);
  }
}

// ---- 2-D path: per-cell register accumulation ------------------------------
// Tiles of 8 x 8 cells.  A CTA takes the points of one work item in batches
// of kBatch2; each batch is counting-sorted by cell in shared memory and its
// 2 x NT1 tap weights and scaled channel values are cached there.  A warp
// then takes one tile row l0 and a block of channel groups: lane
// (jy, group) walks the points of that row cell by cell and sums, in
// registers, the contributions of tap row jy to the NT1 + 7 cells of halo row
// l0 + jy that the 8 cells of the row reach, for kUnitCh channels.  Only
// those sums reach the shared tile (one atomic each), instead of one atomic
// per (point, tap, channel).  In the fixed-point accumulator every product
// is rounded to an integer before it is added, so sums stay exact and the
// grid does not depend on the order of the points.
constexpr int kT2 = 8;         // tile edge of the 2-D path
constexpr int kBatch2 = 256;   // points per batch (one per thread while caching)
constexpr int kUnitCh = 2;     // channels per lane

// Register accumulators hold doubles in both precisions.  Fixed point: each
// product is rounded to the nearest integer (ties to even, like
// __double2ll_rn) by adding and subtracting 1.5 * 2^52 (exact for
// |v| < 2^51), and the integer sums stay below 2^50, so every addition is
// exact; the flush converts the exact integer sum once.
template <typename Acc>
__device__ __forceinline__ void reg_add(double& a, double v);
template <>
__device__ __forceinline__ void reg_add<long long>(double& a, double v) {
  constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
  a = __dadd_rn(a, __dsub_rn(__dadd_rn(v, kRound), kRound));
}
template <>
__device__ __forceinline__ void reg_add<double>(double& a, double v) {
  a += v;
}

template <typename Acc>
__device__ __forceinline__ Acc reg_value(double a);
template <>
__device__ __forceinline__ long long reg_value<long long>(double a) {
  return __double2ll_rn(a);
}
template <>
__device__ __forceinline__ double reg_value<double>(double a) {
  return a;
}

__device__ __forceinline__ void shared_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}
__device__ __forceinline__ void shared_add(double* p, double v) { atomicAdd(p, v); }

// Register accumulators of the 2-D path.  Fixed point: the product v w is
// rounded once to the nearest integer by the fused multiply-add
// t = v w + 1.5 * 2^52 (every double in [2^52, 2^53) is an integer, and
// |v w| < 2^50 keeps t there), and the bit pattern of t is
// bits(1.5 * 2^52) + round(v w), so the register adds the bit patterns in
// integer arithmetic (modulo 2^64) and the flush subtracts the bias once per
// add it received.  One FP64 instruction per product; the sum is exact and
// independent of the order of the points.  Float64 accumulation adds the
// fused product.
template <typename Acc>
struct Reg2;
template <>
struct Reg2<long long> {
  using T = unsigned long long;
  static constexpr unsigned long long kBias = 0x4338000000000000ull;  // bits(1.5 * 2^52)
  __device__ static void add(T& a, double v, double w) {
    a += (unsigned long long)__double_as_longlong(__fma_rn(v, w, 6755399441055744.0));
  }
  __device__ static long long value(T a, int adds) {
    return (long long)(a - (unsigned long long)adds * kBias);
  }
};
template <>
struct Reg2<double> {
  using T = double;
  __device__ static void add(T& a, double v, double w) { a = __fma_rn(v, w, a); }
  __device__ static double value(T a, int) { return a; }
};

// Halo-row stride (odd) and channel stride (odd) of the shared tile.
__host__ __device__ constexpr int row_stride2(int nt1) { return (kT2 + nt1 - 1) | 1; }
__host__ __device__ constexpr int chan_stride2(int w0, int nt1) { return (w0 * row_stride2(nt1)) | 1; }

template <typename Acc, int NT1>
__global__ void __launch_bounds__(kBatch2, 2)
tile_accumulate_2d_kernel(SpreadGeom g, int64_t n, int nchan, int ones_channel, int cgroup,
                          const int* __restrict__ offsets, const int* __restrict__ items,
                          const int* __restrict__ rec_base, const double* __restrict__ rec_frac,
                          const double* __restrict__ rec_val, const double* __restrict__ absum,
                          int margin_bits, Acc* __restrict__ gacc) {
  constexpr int MSP = (NT1 - 1) / 2;
  constexpr int NACC = kT2 + NT1 - 1;  // halo cells one tile row reaches
  constexpr int RS = row_stride2(NT1);
  constexpr int GPL = 32 / NT1;        // channel groups per warp
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int cnt[kT2 * kT2];
  __shared__ int off[kT2 * kT2 + 1];
  __shared__ double scale[32];
  const int c_begin = blockIdx.y * cgroup;
  const int nc = min(nchan, c_begin + cgroup) - c_begin;
  const int T0 = g.T[0], W0 = g.W[0];
  const int CS = chan_stride2(W0, NT1);
  Acc* acc = reinterpret_cast<Acc*>(smem_raw);                       // nc x CS
  double* wy = reinterpret_cast<double*>(acc + (size_t)nc * CS);     // kBatch2 x NT1
  double* wx = wy + kBatch2 * NT1;                                   // kBatch2 x NT1
  double* vs = wx + kBatch2 * NT1;                                   // kBatch2 x nc

  const int item = blockIdx.x;
  if (item >= items[g.ntiles]) return;
  int lo = 0, hi = g.ntiles;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (items[mid] <= item) lo = mid; else hi = mid;
  }
  const int tile = lo;
  const int p_begin = offsets[tile] + (item - items[tile]) * g.item_points;
  const int p_end = min(offsets[tile + 1], p_begin + g.item_points);
  const int tc0 = tile / g.ntile[1], tc1 = tile - tc0 * g.ntile[1];

  for (int i = threadIdx.x; i < nc * CS; i += blockDim.x) acc[i] = Acc(0);
  if (threadIdx.x < 32)
    scale[threadIdx.x] =
        (threadIdx.x < nc && absum != nullptr) ? fixed_scale(absum[c_begin + threadIdx.x], margin_bits)
                                               : 1.0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int jy = lane % NT1, gsub = lane / NT1;
  const int ngrp = (nc + kUnitCh - 1) / kUnitCh;
  const int ngblk = (ngrp + GPL - 1) / GPL;
  const int nlc = T0 * kT2;
  const double hx0 = g.ax[0].hx, hx1 = g.ax[1].hx;
  const double ft0 = g.four_tau[0], ft1 = g.four_tau[1];

  for (int b0 = p_begin; b0 < p_end; b0 += kBatch2) {
    const int nb = min(kBatch2, p_end - b0);
    __syncthreads();  // previous batch's readers are done
    for (int i = threadIdx.x; i < nlc; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    const int q = threadIdx.x;
    int lc = 0, rank = 0;
    if (q < nb) {
      const int packed = rec_base[b0 + q];
      lc = (packed & 1023) * kT2 + ((packed >> 10) & 1023);
      rank = atomicAdd(&cnt[lc], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the <= 64 cell counts
      const int i0 = 2 * lane, i1 = 2 * lane + 1;
      const int a0 = i0 < nlc ? cnt[i0] : 0, a1 = i1 < nlc ? cnt[i1] : 0;
      int incl = a0 + a1;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const int excl = incl - a0 - a1;
      if (i0 < nlc) off[i0] = excl;
      if (i1 < nlc) off[i1] = excl + a0;
      if (lane == 31) off[nlc] = incl;
    }
    __syncthreads();
    if (q < nb) {
      const int pos = off[lc] + rank;
      const int p = b0 + q;
      const double f0 = rec_frac[p], f1 = rec_frac[n + p];
#pragma unroll 1
      for (int j = 0; j < NT1; ++j) {
        const double d0 = f0 - hx0 * (double)(j - MSP);
        const double d1 = f1 - hx1 * (double)(j - MSP);
        wy[pos * NT1 + j] = exp(-(d0 * d0) / ft0);
        wx[pos * NT1 + j] = exp(-(d1 * d1) / ft1);
      }
      for (int c = 0; c < nc; ++c) {
        const int ch = c_begin + c;
        const double v = (ones_channel && ch == 0) ? 1.0 : rec_val[(int64_t)(ch - ones_channel) * n + p];
        vs[pos * nc + c] = v * scale[c];
      }
    }
    __syncthreads();
    // warp items: (tile row l0, block of GPL channel groups)
    for (int wi = warp; wi < T0 * ngblk; wi += nwarps) {
      const int l0 = wi / ngblk, gb = wi - l0 * ngblk;
      const int grp = gb * GPL + gsub;
      const bool active = lane < NT1 * GPL && grp < ngrp;
      const int c0 = grp * kUnitCh;
      typename Reg2<Acc>::T a[kUnitCh][NACC];
#pragma unroll
      for (int k = 0; k < kUnitCh; ++k)
#pragma unroll
        for (int j = 0; j < NACC; ++j) a[k][j] = 0;
      const int rowbase = l0 * kT2;
#pragma unroll
      for (int cr = 0; cr < kT2; ++cr) {
        const int pe = off[rowbase + cr + 1];
#pragma unroll 1
        for (int pp = off[rowbase + cr]; pp < pe; ++pp) {
          const double wyv = wy[pp * NT1 + jy];
          double v[kUnitCh];
#pragma unroll
          for (int k = 0; k < kUnitCh; ++k)
            v[k] = (active && c0 + k < nc) ? wyv * vs[pp * nc + c0 + k] : 0.0;
#pragma unroll
          for (int jx = 0; jx < NT1; ++jx) {
            const double w = wx[pp * NT1 + jx];
#pragma unroll
            for (int k = 0; k < kUnitCh; ++k) Reg2<Acc>::add(a[k][cr + jx], v[k], w);
          }
        }
      }
      if (active) {
        // adds register j received: one per point of the cell rows cr with
        // 0 <= j - cr < NT1
        int rows[kT2];
#pragma unroll
        for (int cr = 0; cr < kT2; ++cr) rows[cr] = off[rowbase + cr + 1] - off[rowbase + cr];
        Acc* rowp = acc + (size_t)(l0 + jy) * RS;
#pragma unroll
        for (int j = 0; j < NACC; ++j) {
          int adds = 0;
#pragma unroll
          for (int cr = 0; cr < kT2; ++cr)
            if (j - cr >= 0 && j - cr < NT1) adds += rows[cr];
#pragma unroll
          for (int k = 0; k < kUnitCh; ++k) {
            if (c0 + k < nc) {
              const Acc val = Reg2<Acc>::value(a[k][j], adds);
              if (val != Acc(0)) shared_add(rowp + (size_t)(c0 + k) * CS + j, val);
            }
          }
        }
      }
    }
  }
  __syncthreads();

  // flush: one global atomic per non-zero cell of the tile + halo
  const int W1 = g.W[1];
  for (int idx = threadIdx.x; idx < nc * W0 * W1; idx += blockDim.x) {
    const int c = idx / (W0 * W1);
    const int r = idx - c * (W0 * W1);
    const int r0 = r / W1, r1 = r - r0 * W1;
    const Acc v = acc[(size_t)c * CS + r0 * RS + r1];
    if (v == Acc(0)) continue;
    int gc0 = (tc0 * kT2 + r0 - g.msp) % g.L[0];
    if (gc0 < 0) gc0 += g.L[0];
    int gc1 = (tc1 * kT2 + r1 - g.msp) % g.L[1];
    if (gc1 < 0) gc1 += g.L[1];
    AccOps<Acc>::add_global(&gacc[(int64_t)(c_begin + c) * g.cells + (int64_t)gc0 * g.L[1] + gc1], v);
  }
}

// ---- 3-D path: column ownership ------------------------------------------
// Tiles of 8 x 8 x 8 cells, halo width W = 7 + NT1 (16 for 9 taps).  Thread
// t of a CTA owns the halo column (x0, x1) = (t / W, t % W) and holds its W
// cells along the last axis in registers.  The points of the work item go in
// batches of kBatch3: their base cells and per-axis tap weights are staged
// in shared memory, the last axis's already times the channel value and the
// fixed-point scale; then every thread walks the batch and adds, for each
// point whose tap footprint covers its column, the NT1 taps along the last
// axis into its registers: (e0 e1) (e2 v scale), rounded to an integer and
// summed exactly, so the grid does not depend on the order of the points
// (no shared atomics).  The lanes of a warp take the same point, so the
// footprint's offset along the last axis is the same for the whole warp.
// One channel at a time (blockIdx.y).
constexpr int kBatch3 = 128;
constexpr int kThreads3 = 256;

inline size_t smem_3d(int nt1) {
  return (size_t)kBatch3 * 3 * nt1 * sizeof(double) + (size_t)kBatch3 * sizeof(int);
}

template <typename Acc, int NT1, int BZ>
__device__ __forceinline__ void column_taps(double (&acc)[7 + NT1], double wxy,
                                            const double* __restrict__ e2v) {
#pragma unroll
  for (int k = 0; k < NT1; ++k) reg_add<Acc>(acc[BZ + k], __dmul_rn(wxy, e2v[k]));
}

template <typename Acc, int NT1, int BZ = 0>
__device__ __forceinline__ void column_dispatch(int bz, double (&acc)[7 + NT1], double wxy,
                                                const double* e2v) {
  if constexpr (BZ < 8) {
    if (bz == BZ)
      column_taps<Acc, NT1, BZ>(acc, wxy, e2v);
    else
      column_dispatch<Acc, NT1, BZ + 1>(bz, acc, wxy, e2v);
  }
}

template <typename Acc, int NT1>
__global__ void __launch_bounds__(kThreads3)
tile_columns_3d_kernel(SpreadGeom g, int64_t n, int ones_channel, const int* __restrict__ offsets,
                       const int* __restrict__ items, const int* __restrict__ rec_base,
                       const double* __restrict__ rec_frac, const double* __restrict__ rec_val,
                       const double* __restrict__ absum, int margin_bits,
                       Acc* __restrict__ gacc) {
  constexpr int MSP = (NT1 - 1) / 2;
  constexpr int W = 7 + NT1;
  constexpr int PP = 3 * NT1;  // per-axis weights of one point
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s_w = reinterpret_cast<double*>(smem_raw);  // [kBatch3][PP]
  int* s_base = reinterpret_cast<int*>(s_w + kBatch3 * PP);
  const int ch = blockIdx.y;
  const int item = blockIdx.x;
  if (item >= items[g.ntiles]) return;
  int lo = 0, hi = g.ntiles;  // tile owning this item: largest t with items[t] <= item
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (items[mid] <= item) lo = mid; else hi = mid;
  }
  const int tile = lo;
  const int p_begin = offsets[tile] + (item - items[tile]) * g.item_points;
  const int p_end = min(offsets[tile + 1], p_begin + g.item_points);
  const double sc = absum ? (double)fixed_scale(absum[ch], margin_bits) : 1.0;
  const bool ones = ones_channel && ch == 0;
  const double* vals = ones ? nullptr : rec_val + (int64_t)(ch - ones_channel) * n;

  const int t = threadIdx.x;
  const bool owner = t < W * W;
  const int c0 = t / W, c1 = t - (t / W) * W;
  double acc[W];
#pragma unroll
  for (int z = 0; z < W; ++z) acc[z] = 0.0;

  for (int b0 = p_begin; b0 < p_end; b0 += kBatch3) {
    const int nb = min(kBatch3, p_end - b0);
    for (int i = t; i < nb * PP; i += blockDim.x) {
      const int pp = i / PP;
      const int r = i - pp * PP;
      const int a = r / NT1, j = r - a * NT1;
      const double fr = rec_frac[(int64_t)a * n + b0 + pp];
      const double diff = fr - g.ax[a].hx * (double)(j - MSP);
      double e = fexp(-(diff * diff) / g.four_tau[a]);
      if (a == 2) {
        // last axis: times the channel value and the fixed-point scale
        if (!ones) e = __dmul_rn(e, vals[b0 + pp]);
        if (sc != 1.0) e = __dmul_rn(e, sc);
      }
      s_w[i] = e;
    }
    for (int i = t; i < nb; i += blockDim.x) s_base[i] = rec_base[b0 + i];
    __syncthreads();
    if (owner) {
      for (int pp = 0; pp < nb; ++pp) {
        const int packed = s_base[pp];
        const int d0 = c0 - (packed & 1023);
        const int d1 = c1 - ((packed >> 10) & 1023);
        if (d0 >= 0 && d0 < NT1 && d1 >= 0 && d1 < NT1) {
          const double* wp = s_w + pp * PP;
          const double wxy = __dmul_rn(wp[d0], wp[NT1 + d1]);
          column_dispatch<Acc, NT1>((packed >> 20) & 1023, acc, wxy, wp + 2 * NT1);
        }
      }
    }
    __syncthreads();  // the next batch overwrites the staged points
  }
  if (!owner) return;
  int tcoord[3];
  {
    int r = tile;
    for (int a = 2; a >= 0; --a) {
      tcoord[a] = r % g.ntile[a];
      r /= g.ntile[a];
    }
  }
  int gc0 = (tcoord[0] * g.T[0] + c0 - g.msp) % g.L[0];
  if (gc0 < 0) gc0 += g.L[0];
  int gc1 = (tcoord[1] * g.T[1] + c1 - g.msp) % g.L[1];
  if (gc1 < 0) gc1 += g.L[1];
  Acc* base = gacc + (int64_t)ch * g.cells + ((int64_t)gc0 * g.L[1] + gc1) * g.L[2];
#pragma unroll
  for (int z = 0; z < W; ++z) {
    if (acc[z] == 0.0) continue;
    int gc2 = (tcoord[2] * g.T[2] + z - g.msp) % g.L[2];
    if (gc2 < 0) gc2 += g.L[2];
    AccOps<Acc>::add_global(base + gc2, reg_value<Acc>(acc[z]));
  }
}

static size_t smem_2d(int W0, int nt1, int cg) {
  return sizeof(double) * ((size_t)cg * chan_stride2(W0, nt1) + (size_t)kBatch2 * (2 * nt1 + cg));
}

// Grid value = accumulator / fixed-point scale (a power of two, so the
// product with its inverse is exact) / n.  Thread per cell, all channels.
template <typename Acc, typename Out, bool kFixed>
__global__ void finalize_kernel(int nchan, int64_t cells, const Acc* __restrict__ gacc,
                                const double* __restrict__ absum, int margin_bits, double inv_n,
                                Out* __restrict__ out) {
  __shared__ double inv_scale[FLPR_MAX_CHANNELS];
  for (int c = threadIdx.x; c < nchan; c += blockDim.x)
    inv_scale[c] = kFixed ? 1.0 / fixed_scale(absum[c], margin_bits) : 1.0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cells;
       i += (int64_t)gridDim.x * blockDim.x) {
    for (int c = 0; c < nchan; ++c) {
      const int64_t k = (int64_t)c * cells + i;
      const double v = (double)gacc[k] * inv_scale[c];
      out[k] = (Out)(v * inv_n);
    }
  }
}

// 2-D grids of at least 8 x 8 cells take the per-cell register path.
static bool use_2d_path(int d, const int* L, int msp) {
  return d == 2 && L[0] >= kT2 && L[1] >= kT2 && 2 * msp + 1 <= 13;
}

static void make_geom(SpreadGeom& g, int d, const int* L, int msp, const double* tau,
                      const double* kmap) {
  memset(&g, 0, sizeof(g));
  const bool path2 = use_2d_path(d, L, msp);
  g.d = d;
  g.msp = msp;
  g.ntaps1 = 2 * msp + 1;
  g.item_points = tuning(FLPR_TUNE_SPREAD_ITEM_POINTS);
  static const int tile2[3] = {16, 16, 1};
  static const int tile3[3] = {8, 8, 8};
  g.cells = 1;
  g.tile_cells = 1;
  g.ntiles = 1;
  for (int a = 0; a < 3; ++a) {
    if (a < d) {
      g.L[a] = L[a];
      int T = d == 1 ? 256 : (d == 2 ? (path2 ? kT2 : tile2[a]) : tile3[a]);
      if (d == 3) {
        // wide stencils (oversampled accuracies): smaller tiles, so that one
        // channel's tile plus halo fits shared memory
        const size_t kMax3 = (size_t)200 * 1024;
        while (T > 1 && sizeof(long long) * (size_t)(T + 2 * msp) * (T + 2 * msp) *
                                (T + 2 * msp) > kMax3)
          T >>= 1;
      }
      if (T > L[a]) T = L[a];
      g.T[a] = T;
      g.ntile[a] = (L[a] + T - 1) / T;
      g.W[a] = T + 2 * msp;
      g.cells *= L[a];
      g.tile_cells *= g.W[a];
      g.ntiles *= g.ntile[a];
      g.four_tau[a] = 4.0 * tau[a];
      const double* k = kmap + 9 * a;
      g.ax[a] = KnotAxis{k[0], k[1], k[2], k[3], k[4], k[5], k[6], k[7], k[8]};
    } else {
      g.L[a] = 1;
      g.T[a] = 1;
      g.ntile[a] = 1;
      g.W[a] = 1;
    }
  }
}

static int margin_bits_for(const SpreadGeom& g) {
  int m = 1;
  for (int a = 0; a < g.d; ++a)
    if (g.L[a] < g.ntaps1) m += 4;  // taps wrap onto the same cell
  return m;
}

static int channel_group(const SpreadGeom& g, int nchan, size_t acc_bytes) {
  // 1-D/2-D: four CTAs per SM; 3-D tiles are larger: two CTAs per SM, or
  // one when a wide stencil's tile needs more
  size_t budget = (g.d == 3 ? 110 : 55) * 1024;
  if (g.d == 3 && acc_bytes * (size_t)g.tile_cells > budget) budget = (size_t)200 * 1024;
  int cg = (int)(budget / (acc_bytes * (size_t)g.tile_cells));
  if (cg > 32) cg = 32;  // fixed-point scales of one group live in 32 shared slots
  if (cg > nchan) cg = nchan;
  return cg;
}

static int channel_group_2d(const SpreadGeom& g, int nchan) {
  // two CTAs per SM
  int cg = nchan < 32 ? nchan : 32;
  while (cg > 1 && smem_2d(g.W[0], g.ntaps1, cg) > (size_t)110 * 1024) --cg;
  return cg;
}

struct SpreadWs {
  int* point_tile;
  int* counts;
  int* offsets;
  int* items;
  int* cursor;
  int* rec_base;
  int* rec_idx;
  void* rec_frac;
  void* rec_val;
  double* absum;
  void* gacc;
};

template <typename A>
static void spread_layout(A& ar, int d, int64_t n, int ntiles, int nchan, int64_t cells,
                          size_t real_bytes, SpreadWs* w) {
  auto p0 = ar.template take<int>(n);
  auto p1 = ar.template take<int>(ntiles);
  auto p2 = ar.template take<int>(ntiles + 1);
  auto p3 = ar.template take<int>(ntiles + 1);
  auto p4 = ar.template take<int>(ntiles);
  auto p5 = ar.template take<int>(n);
  auto p6 = ar.template take<char>((size_t)d * n * real_bytes);
  auto p7 = ar.template take<char>((size_t)(nchan > 1 ? nchan - 1 : 1) * n * real_bytes);
  auto p8 = ar.template take<double>(FLPR_MAX_CHANNELS);
  auto p9 = ar.template take<double>((size_t)nchan * cells);
  auto p10 = ar.template take<int>(n);
  if (w) {
    w->point_tile = (int*)p0;
    w->counts = (int*)p1;
    w->offsets = (int*)p2;
    w->items = (int*)p3;
    w->cursor = (int*)p4;
    w->rec_base = (int*)p5;
    w->rec_frac = (void*)p6;
    w->rec_val = (void*)p7;
    w->absum = (double*)p8;
    w->gacc = (void*)p9;
    w->rec_idx = (int*)p10;
  }
}

struct SizeArena {
  size_t used = 0;
  template <typename T>
  T* take(size_t count) {
    used = align_up(used) + align_up(count * sizeof(T));
    return nullptr;
  }
};

template <int NT1>
static int launch_accumulate(const SpreadGeom& g, int64_t n, int nchan, int ones_channel, int cg,
                             const SpreadWs& w, bool fixed, int margin, size_t smem, dim3 grid,
                             cudaStream_t s) {
  if (fixed) {
    auto k = tile_accumulate_kernel<long long, double, NT1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    FLPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
    k<<<grid, kSpreadThreads, smem, s>>>(g, n, nchan, ones_channel, cg, w.offsets, w.items,
                                         w.rec_base, (const double*)w.rec_frac,
                                         (const double*)w.rec_val, w.absum, margin,
                                         (long long*)w.gacc);
  } else {
    auto k = tile_accumulate_kernel<double, double, NT1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    FLPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
    k<<<grid, kSpreadThreads, smem, s>>>(g, n, nchan, ones_channel, cg, w.offsets, w.items,
                                         w.rec_base, (const double*)w.rec_frac,
                                         (const double*)w.rec_val, nullptr, margin,
                                         (double*)w.gacc);
  }
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int NT1>
static int launch_accumulate_2d(const SpreadGeom& g, int64_t n, int nchan, int ones_channel,
                                int cg, const SpreadWs& w, bool fixed, int margin, dim3 grid,
                                cudaStream_t s) {
  const size_t smem = smem_2d(g.W[0], NT1, cg);
  if (fixed) {
    auto k = tile_accumulate_2d_kernel<long long, NT1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    FLPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
    k<<<grid, kBatch2, smem, s>>>(g, n, nchan, ones_channel, cg, w.offsets, w.items, w.rec_base,
                                  (const double*)w.rec_frac, (const double*)w.rec_val, w.absum,
                                  margin, (long long*)w.gacc);
  } else {
    auto k = tile_accumulate_2d_kernel<double, NT1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    FLPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
    k<<<grid, kBatch2, smem, s>>>(g, n, nchan, ones_channel, cg, w.offsets, w.items, w.rec_base,
                                  (const double*)w.rec_frac, (const double*)w.rec_val, nullptr,
                                  margin, (double*)w.gacc);
  }
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}


// The column kernel covers 3-D tiles of 8^3 with at most 9 taps per axis
// (halo columns fit one CTA of 256 threads).
static bool use_3d_columns(const SpreadGeom& g) {
  if (g.d != 3 || g.ntaps1 > 9) return false;
  for (int a = 0; a < 3; ++a)
    if (g.T[a] != 8 || g.W[a] != 7 + g.ntaps1) return false;
  return true;
}

template <int NT1>
static int launch_columns_3d(const SpreadGeom& g, int64_t n, int nchan, int ones_channel,
                             const SpreadWs& w, bool fixed, int margin, dim3 grid,
                             cudaStream_t s) {
  const size_t smem = smem_3d(NT1);
  if (fixed) {
    auto k = tile_columns_3d_kernel<long long, NT1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    k<<<grid, kThreads3, smem, s>>>(g, n, ones_channel, w.offsets, w.items, w.rec_base,
                                    (const double*)w.rec_frac, (const double*)w.rec_val, w.absum,
                                    margin, (long long*)w.gacc);
  } else {
    auto k = tile_columns_3d_kernel<double, NT1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    k<<<grid, kThreads3, smem, s>>>(g, n, ones_channel, w.offsets, w.items, w.rec_base,
                                    (const double*)w.rec_frac, (const double*)w.rec_val, nullptr,
                                    margin, (double*)w.gacc);
  }
  (void)nchan;
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

static int finalize(const SpreadGeom& g, int64_t n, int nchan, bool fixed, int margin,
                    const SpreadWs& w, void* d_grid_out, cudaStream_t s);

}  // namespace flpr

using namespace flpr;

extern "C" {

size_t flpr_spread_ws(int d, int64_t n, const int* h_L, int msp, int nchan, int prec) {
  if (d < 1 || d > 3 || n < 1 || nchan < 1) return 0;
  SpreadGeom g;
  double tau[3] = {1, 1, 1}, kmap[27] = {0};
  make_geom(g, d, h_L, msp, tau, kmap);
  SizeArena ar;
  spread_layout(ar, d, n, g.ntiles, nchan, g.cells, 8, nullptr);
  return ar.used;
}

// d_kmap: when not null, the knot maps (d x 9) are read on the device from
// there (h_kmap then only supplies the knot spacings, column 8).
static int spread_impl(int d, int64_t n, const double* d_x, const double* h_kmap,
                       const double* d_kmap, const int* h_L, int msp, const double* h_tau,
                       int nchan, int ones_channel, const double* const* h_cols,
                       void* d_grid_out, int prec, void* d_ws, size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "spread: d=%d not in [1,3]", d);
  FLPR_CHECK_ARG(n >= 1 && n < (int64_t)1 << 31, "spread: n=%lld out of range", (long long)n);
  FLPR_CHECK_ARG(msp >= 0 && 2 * msp + 1 <= kMaxTaps1, "spread: msp=%d not in [0,12]", msp);
  FLPR_CHECK_ARG(nchan >= 1 && nchan <= FLPR_MAX_CHANNELS, "spread: nchan=%d", nchan);
  FLPR_CHECK_ARG(ones_channel == 0 || ones_channel == 1, "spread: ones_channel must be 0/1");
  FLPR_CHECK_ARG(prec == FLPR_PREC_F32 || prec == FLPR_PREC_F64, "spread: bad precision");
  for (int a = 0; a < d; ++a) FLPR_CHECK_ARG(h_L[a] >= 1, "spread: L[%d]=%d", a, h_L[a]);
  if (ws_bytes < flpr_spread_ws(d, n, h_L, msp, nchan, prec)) {
    set_error("spread: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  cudaStream_t s = as_stream(stream);
  SpreadGeom g;
  make_geom(g, d, h_L, msp, h_tau, h_kmap);
  {
    // few tiles (small 1-D grids): smaller work items, about four per SM
    const int64_t target = 4LL * sm_count();
    if (g.ntiles < target) {
      const int64_t per = (n + target - 1) / target;
      int ip = 256;
      while (ip < per && ip < g.item_points) ip <<= 1;
      if (ip < g.item_points) g.item_points = ip;
    }
  }
  ChanPtrs cp;
  memset(&cp, 0, sizeof(cp));
  for (int c = 0; c < nchan - ones_channel; ++c) cp.col[c] = h_cols[c];
  Arena ar(d_ws, ws_bytes);
  SpreadWs w;
  const bool fixed = (prec == FLPR_PREC_F32);
  spread_layout(ar, d, n, g.ntiles, nchan, g.cells, 8, &w);
  const int margin = margin_bits_for(g);
  const int nv = nchan - ones_channel;
  FLPR_CUDA(cudaMemsetAsync(w.counts, 0, sizeof(int) * g.ntiles, s));
  FLPR_CUDA(cudaMemsetAsync(w.absum, 0, sizeof(double) * FLPR_MAX_CHANNELS, s));
  FLPR_CUDA(cudaMemsetAsync(w.gacc, 0, sizeof(double) * (size_t)nchan * g.cells, s));

  int nb = (int)((n + 255) / 256);
  if (nb > 8 * sm_count()) nb = 8 * sm_count();
  // per-channel sums of |v|: the fixed-point scales of the FP32 grid and of
  // the sorted adjoint deposits (flpr_deposit_sorted) in either precision
  bin_count_kernel<<<nb, 256, 0, s>>>(g, n, d_x, d_kmap, w.point_tile, w.counts, nchan, ones_channel, cp,
                                      w.absum);
  FLPR_LAUNCH_CHECK();
  tile_scan_kernel<<<1, 1024, 0, s>>>(g.ntiles, g.item_points, w.counts, w.offsets, w.items,
                                      w.cursor);
  FLPR_LAUNCH_CHECK();
  // records and tap weights are float64 in both precisions: FP32 weights
  // lose ~1e-6 on the far taps (exponents near 8), which ill-conditioned
  // local systems in sparse corners amplify; only the accumulator differs
  // one point per thread up to 32 CTAs per SM: every thread waits for the
  // slot its cursor atomic returns, so more of them in flight hide it
  int nbs = (int)((n + 255) / 256);
  if (nbs > 32 * sm_count()) nbs = 32 * sm_count();
  bin_scatter_kernel<double><<<nbs, 256, 0, s>>>(g, n, d_x, d_kmap, w.offsets, w.cursor, nv, cp,
                                                w.rec_base, w.rec_idx, (double*)w.rec_frac,
                                                (double*)w.rec_val);
  FLPR_LAUNCH_CHECK();

  int64_t max_items = (int64_t)g.ntiles + (n + g.item_points - 1) / g.item_points;
  if (use_2d_path(d, h_L, msp)) {
    const int cg2 = channel_group_2d(g, nchan);
    FLPR_CHECK_ARG(cg2 >= 1, "spread: tile does not fit shared memory");
    dim3 grid2((unsigned)max_items, (unsigned)((nchan + cg2 - 1) / cg2));
    int st = FLPR_OK;
    switch (g.ntaps1) {
      case 1: st = launch_accumulate_2d<1>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      case 3: st = launch_accumulate_2d<3>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      case 5: st = launch_accumulate_2d<5>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      case 7: st = launch_accumulate_2d<7>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      case 9: st = launch_accumulate_2d<9>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      case 11: st = launch_accumulate_2d<11>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      case 13: st = launch_accumulate_2d<13>(g, n, nchan, ones_channel, cg2, w, fixed, margin, grid2, s); break;
      default: set_error("spread: msp=%d not supported (0..12)", g.msp); return FLPR_ERR_ARG;
    }
    if (st != FLPR_OK) return st;
    return finalize(g, n, nchan, fixed, margin, w, d_grid_out, s);
  }
  if (use_3d_columns(g)) {
    dim3 grid3((unsigned)max_items, (unsigned)nchan);
    int st = FLPR_OK;
    switch (g.ntaps1) {
      case 1: st = launch_columns_3d<1>(g, n, nchan, ones_channel, w, fixed, margin, grid3, s); break;
      case 3: st = launch_columns_3d<3>(g, n, nchan, ones_channel, w, fixed, margin, grid3, s); break;
      case 5: st = launch_columns_3d<5>(g, n, nchan, ones_channel, w, fixed, margin, grid3, s); break;
      case 7: st = launch_columns_3d<7>(g, n, nchan, ones_channel, w, fixed, margin, grid3, s); break;
      case 9: st = launch_columns_3d<9>(g, n, nchan, ones_channel, w, fixed, margin, grid3, s); break;
      default: set_error("spread: msp=%d not supported by the 3-D path", g.msp); return FLPR_ERR_ARG;
    }
    if (st != FLPR_OK) return st;
    return finalize(g, n, nchan, fixed, margin, w, d_grid_out, s);
  }
  const size_t acc_bytes = 8;
  int cg = channel_group(g, nchan, acc_bytes);
  FLPR_CHECK_ARG(cg >= 1, "spread: tile does not fit shared memory");
  int ngroups = (nchan + cg - 1) / cg;
  size_t smem = acc_bytes * (size_t)cg * g.tile_cells;
  dim3 grid((unsigned)max_items, (unsigned)ngroups);
  int status = FLPR_OK;
  switch (g.ntaps1) {
    case 1: status = launch_accumulate<1>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 3: status = launch_accumulate<3>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 5: status = launch_accumulate<5>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 7: status = launch_accumulate<7>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 9: status = launch_accumulate<9>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 11: status = launch_accumulate<11>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 13: status = launch_accumulate<13>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 15: status = launch_accumulate<15>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 17: status = launch_accumulate<17>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 19: status = launch_accumulate<19>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 21: status = launch_accumulate<21>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 23: status = launch_accumulate<23>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    case 25: status = launch_accumulate<25>(g, n, nchan, ones_channel, cg, w, fixed, margin, smem, grid, s); break;
    default: set_error("spread: msp=%d not supported (0..12)", g.msp); return FLPR_ERR_ARG;
  }
  if (status != FLPR_OK) return status;
  return finalize(g, n, nchan, fixed, margin, w, d_grid_out, s);
}

int flpr_spread(int d, int64_t n, const double* d_x, const double* h_kmap, const int* h_L,
                int msp, const double* h_tau, int nchan, int ones_channel,
                const double* const* h_cols, void* d_grid_out, int prec, void* d_ws,
                size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(h_kmap != nullptr, "spread: null knot map");
  return spread_impl(d, n, d_x, h_kmap, nullptr, h_L, msp, h_tau, nchan, ones_channel, h_cols,
                     d_grid_out, prec, d_ws, ws_bytes, stream);
}

int flpr_spread_dkmap(int d, int64_t n, const double* d_x, const double* d_kmap,
                      const double* h_hx, const int* h_L, int msp, const double* h_tau,
                      int nchan, int ones_channel, const double* const* h_cols,
                      void* d_grid_out, int prec, void* d_ws, size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "spread: d=%d not in [1,3]", d);
  FLPR_CHECK_ARG(d_kmap != nullptr && h_hx != nullptr, "spread: null knot map");
  double hk[27] = {0.0};
  for (int a = 0; a < d; ++a) hk[9 * a + 8] = h_hx[a];
  return spread_impl(d, n, d_x, hk, d_kmap, h_L, msp, h_tau, nchan, ones_channel, h_cols,
                     d_grid_out, prec, d_ws, ws_bytes, stream);
}

int flpr_spread_grid64(int d, int64_t n, const int* h_L, int msp, int nchan, const void* d_ws,
                       size_t ws_bytes, double* d_grid64, void* stream) {
  return flpr_spread_grid64_channels(d, n, h_L, msp, nchan, nchan, d_ws, ws_bytes, d_grid64,
                                     stream);
}

int flpr_spread_grid64_channels(int d, int64_t n, const int* h_L, int msp, int nchan, int nout,
                                const void* d_ws, size_t ws_bytes, double* d_grid64,
                                void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "spread_grid64: d=%d not in [1,3]", d);
  FLPR_CHECK_ARG(n >= 1 && nchan >= 1 && nchan <= FLPR_MAX_CHANNELS, "spread_grid64: n/nchan");
  FLPR_CHECK_ARG(nout >= 1 && nout <= nchan, "spread_grid64: nout=%d not in [1, %d]", nout, nchan);
  FLPR_CHECK_ARG(d_ws != nullptr && d_grid64 != nullptr, "spread_grid64: null pointer");
  for (int a = 0; a < d; ++a) FLPR_CHECK_ARG(h_L[a] >= 1, "spread_grid64: L[%d]=%d", a, h_L[a]);
  if (ws_bytes < flpr_spread_ws(d, n, h_L, msp, nchan, FLPR_PREC_F32)) {
    set_error("spread_grid64: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  SpreadGeom g;
  double tau[3] = {1, 1, 1}, kmap[27] = {0};
  make_geom(g, d, h_L, msp, tau, kmap);
  Arena ar(const_cast<void*>(d_ws), ws_bytes);
  SpreadWs w;
  spread_layout(ar, d, n, g.ntiles, nchan, g.cells, 8, &w);
  int64_t fb64 = (g.cells + 255) / 256;
  if (fb64 > 16 * sm_count()) fb64 = 16 * sm_count();
  finalize_kernel<long long, double, true><<<(int)fb64, 256, 0, as_stream(stream)>>>(
      nout, g.cells, (const long long*)w.gacc, w.absum, margin_bits_for(g), 1.0 / (double)n,
      d_grid64);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_knot_map(int d, int64_t n, const double* d_stats, const double* h_ks,
                  const double* h_r0, const double* h_hx, double* d_kmap, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "knot_map: d=%d not in [1,3]", d);
  FLPR_CHECK_ARG(n >= 1, "knot_map: n=%lld", (long long)n);
  FLPR_CHECK_ARG(d_stats && h_ks && h_r0 && h_hx && d_kmap, "knot_map: null pointer");
  KnotConsts kc{};
  for (int a = 0; a < d; ++a) {
    kc.ks[a] = h_ks[a];
    kc.r0[a] = h_r0[a];
    kc.hx[a] = h_hx[a];
  }
  knot_map_kernel<<<1, 32, 0, as_stream(stream)>>>(d, (double)(n - 1), d_stats, kc, d_kmap);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"

namespace flpr {

static int finalize(const SpreadGeom& g, int64_t n, int nchan, bool fixed, int margin,
                    const SpreadWs& w, void* d_grid_out, cudaStream_t s) {
  int64_t fb64 = (g.cells + 255) / 256;
  if (fb64 > 16 * sm_count()) fb64 = 16 * sm_count();
  const int fb = (int)fb64;
  double inv_n = 1.0 / (double)n;
  if (fixed) {
    finalize_kernel<long long, float, true><<<fb, 256, 0, s>>>(nchan, g.cells, (long long*)w.gacc,
                                                         w.absum, margin, inv_n,
                                                         (float*)d_grid_out);
  } else {
    finalize_kernel<double, double, false><<<fb, 256, 0, s>>>(nchan, g.cells, (double*)w.gacc, nullptr,
                                                       margin, inv_n, (double*)d_grid_out);
  }
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // namespace flpr

// ---- adjoint deposits from the tile-sorted records --------------------------
// The dual form of the GCV / Hutchinson sums (see flpr_deposit) needs, per
// cell g of the raw grid, Q[g][c] = sum_i w_ig v_ic and the corner-pair
// weights B of the multilinear stencils.  Here one CTA takes the same work
// item as the spread (the points of one spreading tile, in tile order, with
// their point indices and channel values already in the records) and
// accumulates its deposits in a shared-memory window of the raw grid around
// the tile; the window goes to the global sums with one atomic per non-zero
// cell.  Every contribution is rounded to a 64-bit fixed-point integer
// (quantum 2^-62 of the channel's absolute sum; of n for the pair weights),
// so the sums are exact and do not depend on the order of the points: the
// deposits, and with them the FP32 fit, are bitwise reproducible.  The
// output arrays Q and B hold the integers until the finishing pass turns
// them into doubles in place.
namespace flpr {

constexpr int kDepThreads = 256;
constexpr int kDepHalo = 2;       // raw-grid cells of margin around a spreading tile
constexpr int kDepMaxChan = 32;

struct DepositGeom {
  int G[2];
  double x0[2], dx[2];
  int m0[2];     // spreading cell of raw-grid node 0, per axis (a window hint only)
  int win[2];    // window extent (raw-grid cells) per axis
  int C;         // value channels
  int ones;      // 1: spread channel 0 was the constant (not deposited)
};

__host__ __device__ constexpr int dep_pairs(int D) { return (1 << D) * ((1 << D) + 1) / 2; }

__device__ __forceinline__ double dep_scale(double absum, int extra_bits) {
  if (!(absum > 0.0)) return 1.0;
  int e = 0;
  frexp(absum, &e);  // absum < 2^e
  return ldexp(1.0, 62 - extra_bits - e);
}

template <int D>
__global__ void __launch_bounds__(kDepThreads)
tile_deposit_kernel(SpreadGeom g, DepositGeom dg, int64_t n, const double* __restrict__ x,
                    const int* __restrict__ offsets, const int* __restrict__ items,
                    const int* __restrict__ rec_idx, const double* __restrict__ rec_val,
                    const double* __restrict__ absum, unsigned long long* __restrict__ qacc,
                    unsigned long long* __restrict__ bacc) {
  constexpr int NC = 1 << D;
  constexpr int NP = dep_pairs(D);
  extern __shared__ __align__(16) unsigned long long sacc[];  // window cells x (C + NP)
  __shared__ double s_scale[kDepMaxChan + 1];
  const int C = dg.C, stride = C + NP;
  const int W0 = dg.win[0], W1 = D == 2 ? dg.win[1] : 1;
  const int item = blockIdx.x;
  if (item >= items[g.ntiles]) return;
  int lo = 0, hi = g.ntiles;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (items[mid] <= item) lo = mid; else hi = mid;
  }
  const int tile = lo;
  const int p_begin = offsets[tile] + (item - items[tile]) * g.item_points;
  const int p_end = min(offsets[tile + 1], p_begin + g.item_points);
  // raw-grid window of the tile: node j sits at spreading cell (m0 + j) mod L
  // (the knots are centred on the periodic grid); points whose stencil
  // leaves the window go straight to the global sums
  int org[2] = {0, 0};
  {
    int tc[2] = {tile, 0};
    if (D == 2) {
      tc[0] = tile / g.ntile[1];
      tc[1] = tile - tc[0] * g.ntile[1];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) {
      int j = (tc[a] * g.T[a] - dg.m0[a]) % g.L[a];
      if (j < 0) j += g.L[a];
      org[a] = j - kDepHalo;
    }
  }
  for (int i = threadIdx.x; i < W0 * W1 * stride; i += kDepThreads) sacc[i] = 0ull;
  if (threadIdx.x < C) s_scale[threadIdx.x] = dep_scale(absum[dg.ones + threadIdx.x], 0);
  if (threadIdx.x == 0) s_scale[C] = dep_scale((double)n, 1);  // pair weights: sum <= n
  __syncthreads();
  // batches of kDepThreads points: first one thread per point forms its
  // corner weights and cells (the window cell, or -1 - the global cell when
  // the stencil leaves the window), then the (point, channel) deposits and
  // the pair weights are spread over all threads
  __shared__ double s_w[kDepThreads * (1 << D)];
  __shared__ int s_cell[kDepThreads * (1 << D)];
  for (int b0 = p_begin; b0 < p_end; b0 += kDepThreads) {
    const int nb = min(kDepThreads, p_end - b0);
    if (threadIdx.x < nb) {
      const int p = b0 + threadIdx.x;
      const int64_t i = rec_idx[p];
      int ix[2] = {0, 0};
      double fr[2] = {0.0, 0.0};
#pragma unroll
      for (int a = 0; a < D; ++a) {
        // the clamped cell of interp_optimized.py:60-78 (the fitted values' stencil)
        const double t = (x[i * D + a] - dg.x0[a]) / dg.dx[a];
        if (t < 0.0) {
          ix[a] = 0;
          fr[a] = 0.0;
        } else if (t >= (double)(dg.G[a] - 1)) {
          ix[a] = dg.G[a] - 2;
          fr[a] = 1.0;
        } else {
          ix[a] = (int)t;
          fr[a] = t - (double)ix[a];
        }
      }
      bool inside = true;
#pragma unroll
      for (int a = 0; a < D; ++a) {
        const int l = ix[a] - org[a];
        inside = inside && l >= 0 && l + 1 < dg.win[a];
      }
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double wk = 1.0;
        int gi = 0, li = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) {
          const int bit = (k >> (D - 1 - a)) & 1;
          wk *= bit ? fr[a] : (1.0 - fr[a]);
          gi = gi * dg.G[a] + ix[a] + bit;
          li = li * dg.win[a] + ix[a] + bit - org[a];
        }
        s_w[threadIdx.x * NC + k] = wk;
        s_cell[threadIdx.x * NC + k] = inside ? li : -1 - gi;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nb * (C + 1); e += kDepThreads) {
      const int c = e / nb, t = e - c * nb;
      const double* w = s_w + t * NC;
      const int* cell = s_cell + t * NC;
      if (c < C) {
        const double vs = rec_val[(int64_t)c * n + b0 + t] * s_scale[c];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          const long long q = __double2ll_rn(w[k] * vs);
          if (q == 0) continue;
          if (cell[k] >= 0)
            atomicAdd(&sacc[cell[k] * stride + c], (unsigned long long)q);
          else
            atomicAdd(&qacc[(int64_t)(-1 - cell[k]) * C + c], (unsigned long long)q);
        }
      } else {
        int pr = 0;
#pragma unroll
        for (int k = 0; k < NC; ++k) {
#pragma unroll
          for (int k2 = k; k2 < NC; ++k2, ++pr) {
            const long long q =
                __double2ll_rn((k == k2 ? 1.0 : 2.0) * w[k] * w[k2] * s_scale[C]);
            if (q == 0) continue;
            if (cell[0] >= 0)
              atomicAdd(&sacc[cell[0] * stride + C + pr], (unsigned long long)q);
            else
              atomicAdd(&bacc[(int64_t)(-1 - cell[0]) * NP + pr], (unsigned long long)q);
          }
        }
      }
    }
    __syncthreads();  // the next batch overwrites the point table
  }
  __syncthreads();
  // window -> global sums, one atomic per non-zero entry
  for (int e = threadIdx.x; e < W0 * W1 * stride; e += kDepThreads) {
    const unsigned long long v = sacc[e];
    if (v == 0ull) continue;
    const int cell = e / stride, j = e - cell * stride;
    const int l0 = D == 2 ? cell / W1 : cell, l1 = D == 2 ? cell - l0 * W1 : 0;
    const int g0 = org[0] + l0, g1 = org[1] + l1;
    if (g0 < 0 || g0 >= dg.G[0] || (D == 2 && (g1 < 0 || g1 >= dg.G[1]))) continue;  // stays 0
    const int64_t gc = D == 2 ? (int64_t)g0 * dg.G[1] + g1 : g0;
    if (j < C)
      atomicAdd(&qacc[gc * C + j], v);
    else
      atomicAdd(&bacc[gc * NP + (j - C)], v);
  }
}

// per-block sums of squares of every channel over a fixed range of point
// indices (the columns in their own order: the result does not depend on
// the order of the sorted records); part[b * C + c]
__global__ void sumsq_kernel(int64_t n, int C, ChanPtrs cp, double* __restrict__ part) {
  __shared__ double red[kDepThreads / 32];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  for (int c = 0; c < C; ++c) {
    double sq = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += kDepThreads) {
      const double v = cp.col[c][i];
      sq += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < kDepThreads / 32; ++k) t += red[k];
      part[(int64_t)blockIdx.x * C + c] = t;
    }
  }
}

// integers -> doubles in place (Q (M, C), B (M, NP))
__global__ void deposit_finish_kernel(int64_t M, int C, int NP, const double* __restrict__ absum,
                                      int ones, int64_t n, double* __restrict__ Q,
                                      double* __restrict__ B) {
  __shared__ double inv[kDepMaxChan + 1];
  if (threadIdx.x < C) inv[threadIdx.x] = 1.0 / dep_scale(absum[ones + threadIdx.x], 0);
  if (threadIdx.x == 0) inv[C] = 1.0 / dep_scale((double)n, 1);
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M * C;
       i += (int64_t)gridDim.x * blockDim.x) {
    const long long v = reinterpret_cast<const long long*>(Q)[i];
    Q[i] = (double)v * inv[i % C];
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M * NP;
       i += (int64_t)gridDim.x * blockDim.x) {
    const long long v = reinterpret_cast<const long long*>(B)[i];
    B[i] = (double)v * inv[C];
  }
}

// sq[c] = sum over the items' partials, in item order (one block per channel)
__global__ void deposit_sq_kernel(int nitems, int C, const double* __restrict__ part,
                                  double* __restrict__ sq) {
  __shared__ double sh[256];
  const int c = blockIdx.x;
  double s = 0.0;
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) s += part[(int64_t)it * C + c];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) sq[c] = sh[0];
}

constexpr int kSumsqBlocks = 512;

static int64_t max_items_of(const SpreadGeom& g, int64_t n) {
  return (int64_t)g.ntiles + (n + g.item_points - 1) / g.item_points;
}

}  // namespace flpr

extern "C" {

size_t flpr_deposit_sorted_ws(int d, int64_t n, const int* h_L, int msp, int nchan) {
  if (d < 1 || d > 2 || n < 1 || nchan < 1) return 0;
  SpreadGeom g;
  double tau[3] = {1, 1, 1}, kmap[27] = {0};
  make_geom(g, d, h_L, msp, tau, kmap);
  return align_up(sizeof(double) * (size_t)kSumsqBlocks * (size_t)nchan);
}

int flpr_deposit_sorted(int d, int64_t n, const double* d_x, const int* h_L, int msp, int nchan,
                        int ones_channel, const double* const* h_cols,
                        const void* d_spread_ws, size_t spread_ws_bytes,
                        const double* h_ax, const int* h_G, const int* h_m0, double* d_Q,
                        double* d_B, double* d_sq, void* d_ws, size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d == 1 || d == 2, "deposit_sorted: d=%d (1 or 2)", d);
  FLPR_CHECK_ARG(ones_channel == 0 || ones_channel == 1, "deposit_sorted: ones_channel");
  const int C = nchan - ones_channel;
  FLPR_CHECK_ARG(n >= 1 && C >= 1 && C <= kDepMaxChan, "deposit_sorted: n=%lld C=%d",
                 (long long)n, C);
  FLPR_CHECK_ARG(d_x && h_cols && d_spread_ws && h_ax && h_G && h_m0 && d_Q && d_B && d_sq && d_ws,
                 "deposit_sorted: null pointer");
  for (int a = 0; a < d; ++a)
    FLPR_CHECK_ARG(h_G[a] >= 2 && h_L[a] >= 1, "deposit_sorted: G[%d]=%d", a, h_G[a]);
  if (spread_ws_bytes < flpr_spread_ws(d, n, h_L, msp, nchan, FLPR_PREC_F32) ||
      ws_bytes < flpr_deposit_sorted_ws(d, n, h_L, msp, nchan)) {
    set_error("deposit_sorted: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  cudaStream_t s = as_stream(stream);
  SpreadGeom g;
  double tau[3] = {1, 1, 1}, kmap[27] = {0};
  make_geom(g, d, h_L, msp, tau, kmap);
  {
    // the work items the spread used (it shrinks them on grids with few tiles)
    const int64_t target = 4LL * sm_count();
    if (g.ntiles < target) {
      const int64_t per = (n + target - 1) / target;
      int ip = 256;
      while (ip < per && ip < g.item_points) ip <<= 1;
      if (ip < g.item_points) g.item_points = ip;
    }
  }
  Arena ar(const_cast<void*>(d_spread_ws), spread_ws_bytes);
  SpreadWs w;
  spread_layout(ar, d, n, g.ntiles, nchan, g.cells, 8, &w);
  DepositGeom dg;
  memset(&dg, 0, sizeof(dg));
  int64_t M = 1;
  for (int a = 0; a < d; ++a) {
    dg.G[a] = h_G[a];
    dg.x0[a] = h_ax[2 * a];
    dg.dx[a] = h_ax[2 * a + 1];
    dg.m0[a] = h_m0[a];
    dg.win[a] = g.T[a] + 2 * kDepHalo;
    M *= h_G[a];
  }
  dg.C = C;
  dg.ones = ones_channel;
  const int NP = dep_pairs(d);
  const int wcells = dg.win[0] * (d == 2 ? dg.win[1] : 1);
  const size_t smem = sizeof(unsigned long long) * (size_t)wcells * (size_t)(C + NP);
  FLPR_CHECK_ARG(smem <= (size_t)200 * 1024, "deposit_sorted: window does not fit shared memory");
  FLPR_CUDA(cudaMemsetAsync(d_Q, 0, sizeof(double) * (size_t)M * C, s));
  FLPR_CUDA(cudaMemsetAsync(d_B, 0, sizeof(double) * (size_t)M * NP, s));
  const int64_t nitems = max_items_of(g, n);
  double* part = static_cast<double*>(d_ws);
  ChanPtrs cp;
  memset(&cp, 0, sizeof(cp));
  for (int c = 0; c < C; ++c) cp.col[c] = h_cols[c];
  if (d == 2) {
    auto k = tile_deposit_kernel<2>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    k<<<(unsigned)nitems, kDepThreads, smem, s>>>(
        g, dg, n, d_x, w.offsets, w.items, w.rec_idx, (const double*)w.rec_val, w.absum,
        reinterpret_cast<unsigned long long*>(d_Q), reinterpret_cast<unsigned long long*>(d_B));
  } else {
    auto k = tile_deposit_kernel<1>;
    FLPR_CUDA(raise_dyn_smem(k, smem));
    k<<<(unsigned)nitems, kDepThreads, smem, s>>>(
        g, dg, n, d_x, w.offsets, w.items, w.rec_idx, (const double*)w.rec_val, w.absum,
        reinterpret_cast<unsigned long long*>(d_Q), reinterpret_cast<unsigned long long*>(d_B));
  }
  FLPR_LAUNCH_CHECK();
  int64_t fb = (M * (C > NP ? C : NP) + 255) / 256;
  if (fb > 8 * sm_count()) fb = 8 * sm_count();
  deposit_finish_kernel<<<(int)fb, 256, 0, s>>>(M, C, NP, w.absum, ones_channel, n, d_Q, d_B);
  FLPR_LAUNCH_CHECK();
  sumsq_kernel<<<kSumsqBlocks, kDepThreads, 0, s>>>(n, C, cp, part);
  FLPR_LAUNCH_CHECK();
  deposit_sq_kernel<<<C, 256, 0, s>>>(kSumsqBlocks, C, part, d_sq);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
