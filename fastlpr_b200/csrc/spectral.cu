// Forward FFT of the spread grids, separable kernel-moment spectra and the
// batched spectral multiply + inverse FFT + crop.
#include <cfloat>
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "plans.cuh"

namespace flpr {

template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};

// ---- kernel factors -------------------------------------------------------
struct FactorArgs {
  int d;
  int G[3], L[3];
  int64_t off[3];  // start of axis a in d_F (elements)
  double lo[3], hi[3];
  int H, npow;
};

// One block per (axis, h, pow): sample exp(-u^2/2) u^p / h on the linspace
// grid, zero padded with floor((L-G)/2)+1 leading zeros.
__global__ void factor_sample_kernel(FactorArgs fa, const double* __restrict__ h,
                                     double2* __restrict__ F, double* __restrict__ sum0) {
  const int row = blockIdx.x;  // (a, hi, p)
  const int per_axis = fa.H * fa.npow;
  const int a = row / per_axis;
  const int r = row - a * per_axis;
  const int hidx = r / fa.npow;
  const int p = r - hidx * fa.npow;
  const int G = fa.G[a], L = fa.L[a];
  const int before = (L - G) / 2 + 1;
  const double hv = h[hidx * fa.d + a];
  const double lo = fa.lo[a], hi = fa.hi[a];
  const double step = G > 1 ? (hi - lo) / (double)(G - 1) : 0.0;
  double2* out = F + fa.off[a] + (int64_t)r * L;
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < L; i += blockDim.x) {
    int k = i - before;
    double v = 0.0;
    if (k >= 0 && k < G) {
      double g = (k == G - 1 && G > 1) ? hi : dadd(dmul((double)k, step), lo);
      double u = ddiv(g, hv);
      double e = exp(dmul(-0.5, dmul(u, u)));
      double pw = 1.0;
      for (int q = 0; q < p; ++q) pw = dmul(pw, u);
      v = ddiv(dmul(e, pw), hv);
      if (p == 0) acc += v;
    }
    out[i] = make_double2(v, 0.0);
  }
  if (p == 0) {
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) sum0[a * fa.H + hidx] = sh[0];
  }
}

// ---- products -------------------------------------------------------------
struct ProdDesc {
  int chan;
  int hidx;
  int pw[3];
};

constexpr int kMaxBatch = 128;

struct ProdBatch {
  ProdDesc p[kMaxBatch];
};

struct ConvArgs {
  int d;
  int L[3];
  int G[3];
  int qout[3];
  int H, npow;
  int64_t half;   // elements of one half spectrum
  int64_t cells;  // prod(L)
  int64_t M;      // prod(G)
  int64_t foff[3];
  double scale;
};

template <typename Real>
__global__ void product_kernel(ConvArgs ca, int nb, ProdBatch desc,
                               const typename Cplx<Real>::type* __restrict__ spec,
                               const double2* __restrict__ F,
                               typename Cplx<Real>::type* __restrict__ out) {
  using C = typename Cplx<Real>::type;
  // a batch holds fewer than 2^31 elements (conv_batch budget): 32-bit indices
  const unsigned total = (unsigned)nb * (unsigned)ca.half;
  const unsigned half = (unsigned)ca.half;
  const unsigned Llast_half = ca.L[ca.d - 1] / 2 + 1;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned bu = t / half;
    const int b = (int)bu;
    const unsigned w = t - bu * half;
    const ProdDesc pd = desc.p[b];
    // decode frequency index (row-major, last axis half length)
    int om[3] = {0, 0, 0};
    {
      unsigned r = w;
      unsigned q = r / Llast_half;
      om[ca.d - 1] = (int)(r - q * Llast_half);
      r = q;
      for (int a = ca.d - 2; a >= 0; --a) {
        const unsigned La = ca.L[a];
        q = r / La;
        om[a] = (int)(r - q * La);
        r = q;
      }
    }
    double kr = ca.scale, ki = 0.0;
    for (int a = 0; a < ca.d; ++a) {
      double2 f = F[ca.foff[a] + ((int64_t)pd.hidx * ca.npow + pd.pw[a]) * ca.L[a] + om[a]];
      double nr = kr * f.x - ki * f.y;
      double ni = kr * f.y + ki * f.x;
      kr = nr;
      ki = ni;
    }
    C s = spec[(int64_t)pd.chan * ca.half + w];
    C o;
    o.x = (Real)((double)s.x * kr - (double)s.y * ki);
    o.y = (Real)((double)s.x * ki + (double)s.y * kr);
    out[t] = o;
  }
}

template <typename Real>
__global__ void crop_kernel(ConvArgs ca, int nb, int p0, const Real* __restrict__ full,
                            int add_eps, Real* __restrict__ out) {
  const unsigned M = (unsigned)ca.M;
  const unsigned total = (unsigned)nb * M;
  const double eps = 2.220446049250313e-16;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned bu = t / M;
    const int b = (int)bu;
    const unsigned g0 = t - bu * M;
    unsigned g = g0;
    int gc[3] = {0, 0, 0};
    for (int a = ca.d - 1; a >= 0; --a) {
      const unsigned Ga = ca.G[a];
      const unsigned q = g / Ga;
      gc[a] = (int)(g - q * Ga);
      g = q;
    }
    int64_t src = 0;
    for (int a = 0; a < ca.d; ++a) src = src * ca.L[a] + (gc[a] + ca.qout[a]);
    Real v = full[(int64_t)b * ca.cells + src];
    if (add_eps) v = (Real)((double)v + eps);
    out[(int64_t)(p0 + b) * ca.M + g0] = v;
  }
}

// ---- radial (non-separable) kernels: full-plane spectra ---------------------
// Kernel ids (kernel.py:159-431): 0 gaussian, 1 gaussian_ft, 2 epanechnikov,
// 3 tricube, 4 quartic/biweight, 5 triweight, 6 uniform; all of ||u||^2.
constexpr int kMaxElems = 64;

struct PlaneArgs {
  int d, kid, H, nelem;
  int G[3], L[3], before[3];
  double lo[3], hi[3], step[3];
  int64_t cells;
  int pw[kMaxElems][3];
};

__device__ __forceinline__ double radial_kernel(int kid, double s) {
  const double eps = 2.220446049250313e-16;
  switch (kid) {
    case 0: return ddiv(exp(dmul(-0.5, s)), 2.5066282746310002);   // / sqrt(2 pi)
    case 1: return exp(dmul(-0.5, s));
    case 2: { const double v = dmul(dsub(1.0, s), 0.75); return v > eps ? v : eps; }
    case 3: {
      const double r = sqrt(s);
      const double c = dsub(1.0, pow(r, 3.0));
      const double v = r <= 1.0 ? dmul(70.0 / 81.0, pow(c, 3.0)) : 0.0;
      return v > eps ? v : eps;
    }
    case 4: {
      const double c = dsub(1.0, s);
      const double v = s <= 1.0 ? dmul(15.0 / 16.0, dmul(c, c)) : 0.0;
      return v > eps ? v : eps;
    }
    case 5: {
      const double v = s <= 1.0 ? dmul(35.0 / 32.0, pow(dsub(1.0, s), 3.0)) : 0.0;
      return v > eps ? v : eps;
    }
    default: return sqrt(s) <= 1.0 ? 0.5 : 0.0;
  }
}

// Real planes of items [i0, i0 + nb) (item = elem * H + h): on the
// zero-padded L grid, K(u) prod_a u_a^pw_a / prod_a h_a at the grid point
// (linspace(lo, hi, G) per axis, u = x / h), zero in the padding.
__global__ void kernel_plane_kernel(PlaneArgs pa, int i0, int nb, const double* __restrict__ h,
                                    double* __restrict__ out) {
  const int64_t total = (int64_t)nb * pa.cells;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / pa.cells);
    int64_t r = t - (int64_t)b * pa.cells;
    const int item = i0 + b;
    const int e = item / pa.H, hidx = item - e * pa.H;
    int k[3] = {0, 0, 0};
    bool inside = true;
    for (int a = pa.d - 1; a >= 0; --a) {
      k[a] = (int)(r % pa.L[a]) - pa.before[a];
      r /= pa.L[a];
      inside = inside && k[a] >= 0 && k[a] < pa.G[a];
    }
    double v = 0.0;
    if (inside) {
      double u[3], ssq = 0.0, deth = 1.0;
      for (int a = 0; a < pa.d; ++a) {
        const double g = (k[a] == pa.G[a] - 1 && pa.G[a] > 1) ? pa.hi[a]
                                                              : dadd(dmul((double)k[a], pa.step[a]), pa.lo[a]);
        const double hv = h[hidx * pa.d + a];
        u[a] = ddiv(g, hv);
        ssq = a == 0 ? dmul(u[a], u[a]) : dadd(ssq, dmul(u[a], u[a]));
        deth = dmul(deth, hv);
      }
      v = ddiv(radial_kernel(pa.kid, ssq), deth);
      for (int a = 0; a < pa.d; ++a)
        for (int q = 0; q < pa.pw[e][a]; ++q) v = dmul(v, u[a]);
    }
    out[t] = v;
  }
}

template <typename Real>
__global__ void product_full_kernel(ConvArgs ca, int nb, ProdBatch desc,
                                    const typename Cplx<Real>::type* __restrict__ spec,
                                    const double2* __restrict__ K,
                                    typename Cplx<Real>::type* __restrict__ out) {
  using C = typename Cplx<Real>::type;
  const int64_t total = (int64_t)nb * ca.half;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / ca.half);
    const int64_t w = t - (int64_t)b * ca.half;
    const ProdDesc pd = desc.p[b];
    const double2 k = K[(int64_t)pd.hidx * ca.half + w];  // hidx = elem * H + h here
    const double kr = k.x * ca.scale, ki = k.y * ca.scale;
    const C sv = spec[(int64_t)pd.chan * ca.half + w];
    C o;
    o.x = (Real)((double)sv.x * kr - (double)sv.y * ki);
    o.y = (Real)((double)sv.x * ki + (double)sv.y * kr);
    out[t] = o;
  }
}

// ---- 2-D separable convolution -----------------------------------------------
// The kernel spectrum factors as A0(w0) A1(w1): a column pass (times A0,
// inverse FFT along axis 0, rows q0..q0+G0-1 kept) shared by every product
// with the same (channel, bandwidth, axis-0 exponent), then a row pass per
// product (times A1 and the scale, C2R along axis 1, columns q1..q1+G1-1).
constexpr int kSepMax = 256;  // jobs per column chunk / products per row batch

struct SepJobs {
  int chan[kSepMax], hidx[kSepMax], p0[kSepMax];
};

struct SepProds {
  int job[kSepMax], hidx[kSepMax], p1[kSepMax], out[kSepMax];
};

struct SepArgs {
  int L0, L1, L1h, G0, G1, q0, q1, npow;
  int64_t f1off;  // start of the axis-1 factors in F
  double scale;
};

// colbuf (L0, Jc, L1h) = spec[chan_j](w0, w1) * A0_{h_j, p0_j}(w0)
template <typename Real>
__global__ void sep_colprod_kernel(SepArgs sa, int jc, int nj, SepJobs jobs,
                                   const typename Cplx<Real>::type* __restrict__ spec,
                                   const double2* __restrict__ F,
                                   typename Cplx<Real>::type* __restrict__ col) {
  using C = typename Cplx<Real>::type;
  // sizes here stay below 2^31 (the buffers are bounded by the workspace
  // budget): 32-bit index arithmetic
  const unsigned total = (unsigned)sa.L0 * jc * sa.L1h;
  const int64_t half = (int64_t)sa.L0 * sa.L1h;
  const unsigned L1h = sa.L1h, ujc = jc;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned r = t / L1h;
    const int w1 = (int)(t - r * L1h);
    const unsigned w0u = r / ujc;
    const int j = (int)(r - w0u * ujc);
    const int w0 = (int)w0u;
    C o;
    if (j < nj) {
      const double2 f = F[((int64_t)jobs.hidx[j] * sa.npow + jobs.p0[j]) * sa.L0 + w0];
      const C v = spec[(int64_t)jobs.chan[j] * half + (int64_t)w0 * sa.L1h + w1];
      o.x = (Real)((double)v.x * f.x - (double)v.y * f.y);
      o.y = (Real)((double)v.x * f.y + (double)v.y * f.x);
    } else {
      o.x = (Real)0;
      o.y = (Real)0;
    }
    col[t] = o;
  }
}

// rowbuf (P, G0, L1h) = col(q0 + x0, job_p, w1) * A1_{h_p, p1_p}(w1) * scale
template <typename Real>
__global__ void sep_rowprod_kernel(SepArgs sa, int jc, int np, int pc, SepProds prods,
                                   const typename Cplx<Real>::type* __restrict__ col,
                                   const double2* __restrict__ F,
                                   typename Cplx<Real>::type* __restrict__ row) {
  using C = typename Cplx<Real>::type;
  const unsigned total = (unsigned)pc * sa.G0 * sa.L1h;
  const unsigned L1h = sa.L1h, G0 = sa.G0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned r = t / L1h;
    const int w1 = (int)(t - r * L1h);
    const unsigned pu = r / G0;
    const int x0 = (int)(r - pu * G0);
    const int p = (int)pu;
    C o;
    if (p < np) {
      const double2 f = F[sa.f1off + ((int64_t)prods.hidx[p] * sa.npow + prods.p1[p]) * sa.L1 + w1];
      const double fr = f.x * sa.scale, fi = f.y * sa.scale;
      const C v = col[((int64_t)(sa.q0 + x0) * jc + prods.job[p]) * sa.L1h + w1];
      o.x = (Real)((double)v.x * fr - (double)v.y * fi);
      o.y = (Real)((double)v.x * fi + (double)v.y * fr);
    } else {
      o.x = (Real)0;
      o.y = (Real)0;
    }
    row[t] = o;
  }
}

// out[prod.out][x0 * G1 + x1] = real(q1 + x1) of row (p, x0)
template <typename Real>
__global__ void sep_crop_kernel(SepArgs sa, int np, SepProds prods, const Real* __restrict__ real,
                                int add_eps, Real* __restrict__ out) {
  const unsigned M = (unsigned)sa.G0 * sa.G1;
  const unsigned total = (unsigned)np * M;
  const unsigned G1 = sa.G1;
  const double eps = 2.220446049250313e-16;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned pu = t / M;
    const unsigned g = t - pu * M;
    const unsigned x0u = g / G1;
    const int p = (int)pu;
    const int x0 = (int)x0u, x1 = (int)(g - x0u * G1);
    Real v = real[((int64_t)p * sa.G0 + x0) * sa.L1 + sa.q1 + x1];
    if (add_eps) v = (Real)((double)v + eps);
    out[(int64_t)prods.out[p] * M + g] = v;
  }
}

static int conv_batch(int d, const int* L, int nprod, int prec) {
  int64_t cells = prod(L, d);
  int64_t half = cells / L[d - 1] * (L[d - 1] / 2 + 1);
  size_t es = prec == FLPR_PREC_F32 ? 4 : 8;
  size_t per = (size_t)half * 2 * es + (size_t)cells * es;
  size_t budget = (size_t)1536 << 20;
  int64_t b = (int64_t)(budget / per);
  if (b < 1) b = 1;
  if (b > nprod) b = nprod;
  if (b > kMaxBatch) b = kMaxBatch;
  return (int)b;
}

static int grid_blocks(int64_t total) {
  int64_t b = (total + 255) / 256;
  int64_t cap = 32 * (int64_t)sm_count();
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace flpr

using namespace flpr;

// Oversampled spreading (accuracy >= 7; nufftn_type1.py:693-770 followed by
// the ifftshift of convolution.py:235-236): from the R2C spectrum of the
// ratio*L grid keep the L frequencies f in [-floor(L/2), L - floor(L/2) - 1]
// per axis, divide by ratio^d and by
// Kn = sqrt(prod tau / pi^d) exp(-sum_a tau_a f_a^2), and store them in the
// R2C layout of an L grid (index k <-> f = k for k < (L+1)/2, else k - L).
// The last axis keeps k in [0, L/2]; a negative f there (the Nyquist entry of
// an even L) comes from the Hermitian mirror of the input.
struct OverArgs {
  int d, C;
  int Lo[3], Li[3];
  int64_t half_o, half_i;   // entries per channel
  double tau[3];
  double kn0, inv_rd;
};

// Big-grid spectrum value at frequency g (|g_a| <= Li_a / 2) from its half
// spectrum: negative last-axis frequencies are read at -g, conjugated.
template <typename T2>
__device__ __forceinline__ double2 big_at(const OverArgs& a, const T2* __restrict__ in_c, const int* g) {
  const int d = a.d;
  const bool mirror = g[d - 1] < 0;
  int64_t ii = 0;
  for (int ax = 0; ax < d - 1; ++ax) {
    int fi = mirror ? -g[ax] : g[ax];
    fi %= a.Li[ax];
    if (fi < 0) fi += a.Li[ax];
    ii = ii * a.Li[ax] + fi;
  }
  ii = ii * (a.Li[d - 1] / 2 + 1) + (mirror ? -g[d - 1] : g[d - 1]);
  const T2 v = in_c[ii];
  return make_double2((double)v.x, mirror ? -(double)v.y : (double)v.y);
}

// Output bin f of the L grid (standard order).  The reference keeps the
// cropped full spectrum X and takes the real part after its inverse
// transform, which equals transforming the Hermitian part
// (X[f] + conj(X[-f])) / 2.  That differs from X only where some f_a is the
// even-size Nyquist frequency -L_a/2, whose partner -f_a aliases to the same
// bin; there the Hermitian part is the mean of the big-grid values at -L_a/2
// and +L_a/2, which is what is stored so that the half spectrum is exact.
template <typename T2>
__global__ void oversample_crop_kernel(OverArgs a, const T2* __restrict__ in, T2* __restrict__ out) {
  const int64_t total = (int64_t)a.C * a.half_o;
  const int d = a.d;
  const int Lol = a.Lo[d - 1];
  const int ho = Lol / 2 + 1;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / a.half_o;
    int64_t r = t - c * a.half_o;
    int f[3], fp[3];
    bool nyq = false;
    // last axis (half spectrum), then the others, row-major
    const int kl = (int)(r % ho);
    r /= ho;
    f[d - 1] = kl < (Lol + 1) / 2 ? kl : kl - Lol;
    for (int ax = d - 2; ax >= 0; --ax) {
      const int k = (int)(r % a.Lo[ax]);
      r /= a.Lo[ax];
      f[ax] = k < (a.Lo[ax] + 1) / 2 ? k : k - a.Lo[ax];
    }
    double ex = 0.0;
    for (int ax = 0; ax < d; ++ax) {
      ex += a.tau[ax] * (double)f[ax] * (double)f[ax];
      const bool nq = (a.Lo[ax] % 2 == 0) && f[ax] == -a.Lo[ax] / 2;
      fp[ax] = nq ? -f[ax] : f[ax];
      nyq |= nq;
    }
    double kn = a.kn0 * exp(-ex);
    kn = kn > DBL_MIN ? kn : DBL_MIN;
    const double scale = a.inv_rd / kn;
    const T2* in_c = in + c * a.half_i;
    double2 v = big_at(a, in_c, f);
    if (nyq) {
      const double2 w = big_at(a, in_c, fp);
      v.x = 0.5 * (v.x + w.x);
      v.y = 0.5 * (v.y + w.y);
    }
    T2 o;
    o.x = (decltype(o.x))(v.x * scale);
    o.y = (decltype(o.y))(v.y * scale);
    out[t] = o;
  }
}

extern "C" {

size_t flpr_forward_fft_ws(flpr_handle_t handle, int d, const int* h_L, int nchan, int prec) {
  size_t w = 0;
  PlanKey k = grid_plan(d, h_L, prec == FLPR_PREC_F32 ? CUFFT_R2C : CUFFT_D2Z, nchan);
  if (plans_of(handle).work_size(k, &w) != FLPR_OK) return 0;
  return align_up(w);
}

int flpr_forward_fft(flpr_handle_t handle, int d, const int* h_L, int nchan, void* d_grid,
                     void* d_spec, int prec, void* d_ws, size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "forward_fft: d=%d", d);
  FLPR_CHECK_ARG(nchan >= 1, "forward_fft: nchan=%d", nchan);
  PlanKey k = grid_plan(d, h_L, prec == FLPR_PREC_F32 ? CUFFT_R2C : CUFFT_D2Z, nchan);
  return plans_of(handle).exec(k, d_grid, d_spec, d_ws, ws_bytes, as_stream(stream));
}

static PlanKey factor_plan(int L, int batch) {
  PlanKey k{};
  k.rank = 1;
  k.n[0] = L;
  k.type = CUFFT_Z2Z;
  k.batch = batch;
  k.idist = L;
  k.odist = L;
  return k;
}

size_t flpr_kernel_factors_ws(flpr_handle_t handle, int d, const int* h_L, int H, int npow) {
  size_t mx = 0;
  for (int a = 0; a < d; ++a) {
    size_t w = 0;
    if (plans_of(handle).work_size(factor_plan(h_L[a], H * npow), &w) != FLPR_OK) return 0;
    if (w > mx) mx = w;
  }
  return align_up(mx);
}

int flpr_kernel_factors(flpr_handle_t handle, int d, const int* h_G, const int* h_L,
                        const double* h_lo, const double* h_hi, int H, const double* d_h,
                        int npow, void* d_F, double* d_sum0, void* d_ws, size_t ws_bytes,
                        void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "kernel_factors: d=%d", d);
  FLPR_CHECK_ARG(H >= 1 && npow >= 1 && npow <= 8, "kernel_factors: H=%d npow=%d", H, npow);
  FactorArgs fa{};
  fa.d = d;
  fa.H = H;
  fa.npow = npow;
  int64_t off = 0;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(h_G[a] >= 1 && h_L[a] >= h_G[a] + 1, "kernel_factors: G=%d L=%d", h_G[a],
                   h_L[a]);
    fa.G[a] = h_G[a];
    fa.L[a] = h_L[a];
    fa.lo[a] = h_lo[a];
    fa.hi[a] = h_hi[a];
    fa.off[a] = off;
    off += (int64_t)H * npow * h_L[a];
  }
  cudaStream_t s = as_stream(stream);
  factor_sample_kernel<<<d * H * npow, 256, 0, s>>>(fa, d_h, (double2*)d_F, d_sum0);
  FLPR_LAUNCH_CHECK();
  for (int a = 0; a < d; ++a) {
    double2* base = (double2*)d_F + fa.off[a];
    FLPR_TRY(plans_of(handle).exec(factor_plan(h_L[a], H * npow), base, base, d_ws, ws_bytes, s));
  }
  return FLPR_OK;
}

size_t flpr_conv_ws(flpr_handle_t handle, int d, const int* h_L, int nprod, int prec) {
  if (d < 1 || d > 3 || nprod < 1) return 0;
  int B = conv_batch(d, h_L, nprod, prec);
  int64_t cells = prod(h_L, d);
  int64_t half = cells / h_L[d - 1] * (h_L[d - 1] / 2 + 1);
  size_t es = prec == FLPR_PREC_F32 ? 4 : 8;
  ArenaSize ar;
  ar.take<char>((size_t)B * half * 2 * es);
  ar.take<char>((size_t)B * cells * es);
  int type = prec == FLPR_PREC_F32 ? CUFFT_C2R : CUFFT_Z2D;
  size_t w1 = 0, w2 = 0;
  if (plans_of(handle).work_size(grid_plan(d, h_L, type, B), &w1) != FLPR_OK) return 0;
  int tail = nprod % B;
  if (tail && plans_of(handle).work_size(grid_plan(d, h_L, type, tail), &w2) != FLPR_OK) return 0;
  ar.take<char>(w1 > w2 ? w1 : w2);
  return ar.used;
}

int flpr_conv(flpr_handle_t handle, int d, const int* h_G, const int* h_L, const int* h_qout,
              int H, int npow, const void* d_spec, const void* d_F, int nprod,
              const int* h_chan, const int* h_hidx, const int* h_pow, double scale, int add_eps,
              void* d_out, int prec, void* d_ws, size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "conv: d=%d", d);
  FLPR_CHECK_ARG(nprod >= 1, "conv: nprod=%d", nprod);
  ConvArgs ca{};
  ca.d = d;
  ca.H = H;
  ca.npow = npow;
  ca.scale = scale;
  int64_t off = 0;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(h_qout[a] >= 0 && h_qout[a] + h_G[a] <= h_L[a], "conv: crop window");
    ca.L[a] = h_L[a];
    ca.G[a] = h_G[a];
    ca.qout[a] = h_qout[a];
    ca.foff[a] = off;
    off += (int64_t)H * npow * h_L[a];
  }
  ca.cells = prod(h_L, d);
  ca.M = prod(h_G, d);
  ca.half = ca.cells / h_L[d - 1] * (h_L[d - 1] / 2 + 1);
  for (int p = 0; p < nprod; ++p) {
    FLPR_CHECK_ARG(h_hidx[p] >= 0 && h_hidx[p] < H, "conv: hidx[%d]=%d", p, h_hidx[p]);
    for (int a = 0; a < d; ++a)
      FLPR_CHECK_ARG(h_pow[p * d + a] >= 0 && h_pow[p * d + a] < npow, "conv: pow out of range");
  }
  if (ws_bytes < flpr_conv_ws(handle, d, h_L, nprod, prec)) {
    set_error("conv: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  const int B = conv_batch(d, h_L, nprod, prec);
  FLPR_CHECK_ARG((int64_t)B * ca.cells < ((int64_t)1 << 31),
                 "conv: grid too large for 32-bit batch indexing");
  const size_t es = prec == FLPR_PREC_F32 ? 4 : 8;
  Arena ar(d_ws, ws_bytes);
  char* pbuf = ar.take<char>((size_t)B * ca.half * 2 * es);
  char* rbuf = ar.take<char>((size_t)B * ca.cells * es);
  size_t work_bytes = ar.size - align_up(ar.used);
  char* work = ar.take<char>(1);
  cudaStream_t s = as_stream(stream);
  ProdBatch batch;
  const int ctype = prec == FLPR_PREC_F32 ? CUFFT_C2R : CUFFT_Z2D;
  for (int p0 = 0; p0 < nprod; p0 += B) {
    int nb = nprod - p0 < B ? nprod - p0 : B;
    for (int b = 0; b < nb; ++b) {
      ProdDesc pd{};
      pd.chan = h_chan[p0 + b];
      pd.hidx = h_hidx[p0 + b];
      for (int a = 0; a < 3; ++a) pd.pw[a] = a < d ? h_pow[(p0 + b) * d + a] : 0;
      batch.p[b] = pd;
    }
    int blocks = grid_blocks((int64_t)nb * ca.half);
    if (prec == FLPR_PREC_F32) {
      product_kernel<float><<<blocks, 256, 0, s>>>(ca, nb, batch, (const float2*)d_spec,
                                                   (const double2*)d_F, (float2*)pbuf);
    } else {
      product_kernel<double><<<blocks, 256, 0, s>>>(ca, nb, batch, (const double2*)d_spec,
                                                    (const double2*)d_F, (double2*)pbuf);
    }
    FLPR_LAUNCH_CHECK();
    FLPR_TRY(plans_of(handle).exec(grid_plan(d, h_L, ctype, nb), pbuf, rbuf, work, work_bytes, s));
    int cb = grid_blocks((int64_t)nb * ca.M);
    if (prec == FLPR_PREC_F32) {
      crop_kernel<float><<<cb, 256, 0, s>>>(ca, nb, p0, (const float*)rbuf, add_eps,
                                            (float*)d_out);
    } else {
      crop_kernel<double><<<cb, 256, 0, s>>>(ca, nb, p0, (const double*)rbuf, add_eps,
                                             (double*)d_out);
    }
    FLPR_LAUNCH_CHECK();
  }
  return FLPR_OK;
}


struct SepSizes {
  int jc, pc;
  size_t col_bytes, row_bytes, real_bytes;
};

static SepSizes sep_sizes(const int* G, const int* L, int nprod, int prec) {
  SepSizes z{};
  const size_t es = prec == FLPR_PREC_F32 ? 4 : 8;
  const int L1h = L[1] / 2 + 1;
  const size_t budget = (size_t)256 << 20;
  const size_t per_job = (size_t)L[0] * L1h * 2 * es;
  const size_t per_prod = (size_t)G[0] * (L1h * 2 + L[1]) * es;
  int64_t jc = (int64_t)(budget / per_job), pc = (int64_t)(budget / per_prod);
  z.jc = (int)std::max<int64_t>(1, std::min<int64_t>({jc, (int64_t)kSepMax, (int64_t)nprod}));
  z.pc = (int)std::max<int64_t>(1, std::min<int64_t>({pc, (int64_t)kSepMax, (int64_t)nprod}));
  z.col_bytes = per_job * z.jc;
  z.row_bytes = (size_t)z.pc * G[0] * L1h * 2 * es;
  z.real_bytes = (size_t)z.pc * G[0] * L[1] * es;
  return z;
}

static PlanKey sep_col_plan(const int* L, int jc, int prec) {
  PlanKey k{};
  k.rank = 1;
  k.n[0] = L[0];
  k.type = prec == FLPR_PREC_F32 ? CUFFT_C2C : CUFFT_Z2Z;
  k.batch = jc * (L[1] / 2 + 1);
  k.stride = jc * (L[1] / 2 + 1);
  k.idist = 1;
  k.odist = 1;
  k.inverse = 1;
  return k;
}

static PlanKey sep_row_plan(const int* G, const int* L, int pc, int prec) {
  PlanKey k{};
  k.rank = 1;
  k.n[0] = L[1];
  k.type = prec == FLPR_PREC_F32 ? CUFFT_C2R : CUFFT_Z2D;
  k.batch = pc * G[0];
  k.idist = L[1] / 2 + 1;
  k.odist = L[1];
  return k;
}

size_t flpr_conv2d_sep_ws(flpr_handle_t handle, const int* h_G, const int* h_L, int nprod,
                          int prec) {
  if (nprod < 1) return 0;
  const SepSizes z = sep_sizes(h_G, h_L, nprod, prec);
  size_t w1 = 0, w2 = 0;
  if (plans_of(handle).work_size(sep_col_plan(h_L, z.jc, prec), &w1) != FLPR_OK) return 0;
  if (plans_of(handle).work_size(sep_row_plan(h_G, h_L, z.pc, prec), &w2) != FLPR_OK) return 0;
  ArenaSize ar;
  ar.take<char>(z.col_bytes);
  ar.take<char>(z.row_bytes);
  ar.take<char>(z.real_bytes);
  ar.take<char>(w1 > w2 ? w1 : w2);
  return ar.used;
}

int flpr_conv2d_sep(flpr_handle_t handle, const int* h_G, const int* h_L, const int* h_qout,
                    int H, int npow, const void* d_spec, const void* d_F, int nprod,
                    const int* h_chan, const int* h_hidx, const int* h_pow, double scale,
                    int add_eps, void* d_out, int prec, void* d_ws, size_t ws_bytes,
                    void* stream) {
  FLPR_CHECK_ARG(nprod >= 1 && H >= 1 && npow >= 1, "conv2d_sep: nprod=%d H=%d npow=%d", nprod,
                 H, npow);
  for (int a = 0; a < 2; ++a)
    FLPR_CHECK_ARG(h_qout[a] >= 0 && h_qout[a] + h_G[a] <= h_L[a] && h_G[a] >= 1,
                   "conv2d_sep: crop window");
  for (int p = 0; p < nprod; ++p) {
    FLPR_CHECK_ARG(h_hidx[p] >= 0 && h_hidx[p] < H, "conv2d_sep: hidx[%d]=%d", p, h_hidx[p]);
    FLPR_CHECK_ARG(h_pow[2 * p] >= 0 && h_pow[2 * p] < npow && h_pow[2 * p + 1] >= 0 &&
                       h_pow[2 * p + 1] < npow,
                   "conv2d_sep: pow out of range");
    FLPR_CHECK_ARG(h_chan[p] >= 0, "conv2d_sep: chan[%d]=%d", p, h_chan[p]);
  }
  if (ws_bytes < flpr_conv2d_sep_ws(handle, h_G, h_L, nprod, prec)) {
    set_error("conv2d_sep: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  const SepSizes z = sep_sizes(h_G, h_L, nprod, prec);
  FLPR_CHECK_ARG((int64_t)h_L[0] * z.jc * (h_L[1] / 2 + 1) < ((int64_t)1 << 31) &&
                     (int64_t)z.pc * h_G[0] * h_L[1] < ((int64_t)1 << 31),
                 "conv2d_sep: pass sizes exceed 32-bit indexing");
  SepArgs sa{};
  sa.L0 = h_L[0];
  sa.L1 = h_L[1];
  sa.L1h = h_L[1] / 2 + 1;
  sa.G0 = h_G[0];
  sa.G1 = h_G[1];
  sa.q0 = h_qout[0];
  sa.q1 = h_qout[1];
  sa.npow = npow;
  sa.f1off = (int64_t)H * npow * h_L[0];
  sa.scale = scale;
  Arena ar(d_ws, ws_bytes);
  char* col = ar.take<char>(z.col_bytes);
  char* row = ar.take<char>(z.row_bytes);
  char* real = ar.take<char>(z.real_bytes);
  size_t work_bytes = ar.size - align_up(ar.used);
  char* work = ar.take<char>(1);
  cudaStream_t s = as_stream(stream);
  // column jobs: distinct (channel, bandwidth, axis-0 exponent), first-seen order
  std::vector<int> job_of(nprod);
  std::map<std::tuple<int, int, int>, int> ids;
  std::vector<std::tuple<int, int, int>> jobs;
  for (int p = 0; p < nprod; ++p) {
    auto key = std::make_tuple(h_chan[p], h_hidx[p], h_pow[2 * p]);
    auto it = ids.find(key);
    if (it == ids.end()) {
      it = ids.emplace(key, (int)jobs.size()).first;
      jobs.push_back(key);
    }
    job_of[p] = it->second;
  }
  const int njobs = (int)jobs.size();
  const PlanKey colk = sep_col_plan(h_L, z.jc, prec), rowk = sep_row_plan(h_G, h_L, z.pc, prec);
  std::vector<int> members;
  for (int j0 = 0; j0 < njobs; j0 += z.jc) {
    const int nj = std::min(z.jc, njobs - j0);
    SepJobs sj{};
    for (int j = 0; j < nj; ++j) {
      sj.chan[j] = std::get<0>(jobs[j0 + j]);
      sj.hidx[j] = std::get<1>(jobs[j0 + j]);
      sj.p0[j] = std::get<2>(jobs[j0 + j]);
    }
    const int cb = grid_blocks((int64_t)sa.L0 * z.jc * sa.L1h);
    if (prec == FLPR_PREC_F32)
      sep_colprod_kernel<float><<<cb, 256, 0, s>>>(sa, z.jc, nj, sj, (const float2*)d_spec,
                                                   (const double2*)d_F, (float2*)col);
    else
      sep_colprod_kernel<double><<<cb, 256, 0, s>>>(sa, z.jc, nj, sj, (const double2*)d_spec,
                                                    (const double2*)d_F, (double2*)col);
    FLPR_LAUNCH_CHECK();
    FLPR_TRY(plans_of(handle).exec(colk, col, col, work, work_bytes, s));
    members.clear();
    for (int p = 0; p < nprod; ++p)
      if (job_of[p] >= j0 && job_of[p] < j0 + nj) members.push_back(p);
    for (size_t m0 = 0; m0 < members.size(); m0 += z.pc) {
      const int np = (int)std::min<size_t>(z.pc, members.size() - m0);
      SepProds sp{};
      for (int q = 0; q < np; ++q) {
        const int p = members[m0 + q];
        sp.job[q] = job_of[p] - j0;
        sp.hidx[q] = h_hidx[p];
        sp.p1[q] = h_pow[2 * p + 1];
        sp.out[q] = p;
      }
      const int rb = grid_blocks((int64_t)z.pc * sa.G0 * sa.L1h);
      if (prec == FLPR_PREC_F32)
        sep_rowprod_kernel<float><<<rb, 256, 0, s>>>(sa, z.jc, np, z.pc, sp, (const float2*)col,
                                                     (const double2*)d_F, (float2*)row);
      else
        sep_rowprod_kernel<double><<<rb, 256, 0, s>>>(sa, z.jc, np, z.pc, sp, (const double2*)col,
                                                      (const double2*)d_F, (double2*)row);
      FLPR_LAUNCH_CHECK();
      FLPR_TRY(plans_of(handle).exec(rowk, row, real, work, work_bytes, s));
      const int ob = grid_blocks((int64_t)np * sa.G0 * sa.G1);
      if (prec == FLPR_PREC_F32)
        sep_crop_kernel<float><<<ob, 256, 0, s>>>(sa, np, sp, (const float*)real, add_eps,
                                                  (float*)d_out);
      else
        sep_crop_kernel<double><<<ob, 256, 0, s>>>(sa, np, sp, (const double*)real, add_eps,
                                                   (double*)d_out);
      FLPR_LAUNCH_CHECK();
    }
  }
  return FLPR_OK;
}


static int plane_batch(int d, const int* L, int nitems) {
  int64_t cells = prod(L, d);
  size_t per = (size_t)cells * 8;
  int64_t b = (int64_t)(((size_t)1024 << 20) / per);
  if (b < 1) b = 1;
  if (b > nitems) b = nitems;
  return (int)b;
}

size_t flpr_kernel_spectra_ws(flpr_handle_t handle, int d, const int* h_L, int nitems) {
  if (d < 1 || d > 3 || nitems < 1) return 0;
  const int B = plane_batch(d, h_L, nitems);
  ArenaSize ar;
  ar.take<char>((size_t)B * prod(h_L, d) * 8);
  size_t w1 = 0, w2 = 0;
  if (plans_of(handle).work_size(grid_plan(d, h_L, CUFFT_D2Z, B), &w1) != FLPR_OK) return 0;
  const int tail = nitems % B;
  if (tail && plans_of(handle).work_size(grid_plan(d, h_L, CUFFT_D2Z, tail), &w2) != FLPR_OK)
    return 0;
  ar.take<char>(w1 > w2 ? w1 : w2);
  return ar.used;
}

int flpr_kernel_spectra(flpr_handle_t handle, int d, const int* h_G, const int* h_L,
                        const double* h_lo, const double* h_hi, int kernel_id, int H,
                        const double* d_h, int nelem, const int* h_pow, void* d_K, void* d_ws,
                        size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "kernel_spectra: d=%d", d);
  FLPR_CHECK_ARG(kernel_id >= 0 && kernel_id <= 6, "kernel_spectra: kernel_id=%d", kernel_id);
  FLPR_CHECK_ARG(H >= 1 && nelem >= 1 && nelem <= kMaxElems, "kernel_spectra: H=%d nelem=%d", H,
                 nelem);
  PlaneArgs pa{};
  pa.d = d;
  pa.kid = kernel_id;
  pa.H = H;
  pa.nelem = nelem;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(h_G[a] >= 1 && h_L[a] >= h_G[a] + 1, "kernel_spectra: G=%d L=%d", h_G[a],
                   h_L[a]);
    pa.G[a] = h_G[a];
    pa.L[a] = h_L[a];
    pa.before[a] = (h_L[a] - h_G[a]) / 2 + 1;
    pa.lo[a] = h_lo[a];
    pa.hi[a] = h_hi[a];
    pa.step[a] = h_G[a] > 1 ? (h_hi[a] - h_lo[a]) / (double)(h_G[a] - 1) : 0.0;
  }
  for (int e = 0; e < nelem; ++e)
    for (int a = 0; a < 3; ++a) {
      pa.pw[e][a] = a < d ? h_pow[e * d + a] : 0;
      FLPR_CHECK_ARG(pa.pw[e][a] >= 0 && pa.pw[e][a] <= 8, "kernel_spectra: power out of range");
    }
  pa.cells = prod(h_L, d);
  const int nitems = nelem * H;
  if (ws_bytes < flpr_kernel_spectra_ws(handle, d, h_L, nitems)) {
    set_error("kernel_spectra: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  const int B = plane_batch(d, h_L, nitems);
  const int64_t half = pa.cells / h_L[d - 1] * (h_L[d - 1] / 2 + 1);
  Arena ar(d_ws, ws_bytes);
  double* planes = ar.take<double>((size_t)B * pa.cells);
  size_t work_bytes = ar.size - align_up(ar.used);
  char* work = ar.take<char>(1);
  cudaStream_t s = as_stream(stream);
  for (int i0 = 0; i0 < nitems; i0 += B) {
    const int nb = nitems - i0 < B ? nitems - i0 : B;
    kernel_plane_kernel<<<grid_blocks((int64_t)nb * pa.cells), 256, 0, s>>>(pa, i0, nb, d_h,
                                                                            planes);
    FLPR_LAUNCH_CHECK();
    FLPR_TRY(plans_of(handle).exec(grid_plan(d, h_L, CUFFT_D2Z, nb), planes,
                                   (double2*)d_K + (int64_t)i0 * half, work, work_bytes, s));
  }
  return FLPR_OK;
}

int flpr_conv_full(flpr_handle_t handle, int d, const int* h_G, const int* h_L, const int* h_qout,
                   int nkern, const void* d_spec, const void* d_K, int nprod, const int* h_chan,
                   const int* h_kidx, double scale, int add_eps, void* d_out, int prec,
                   void* d_ws, size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "conv_full: d=%d", d);
  FLPR_CHECK_ARG(nprod >= 1 && nkern >= 1, "conv_full: nprod=%d nkern=%d", nprod, nkern);
  ConvArgs ca{};
  ca.d = d;
  ca.scale = scale;
  for (int a = 0; a < d; ++a) {
    FLPR_CHECK_ARG(h_qout[a] >= 0 && h_qout[a] + h_G[a] <= h_L[a], "conv_full: crop window");
    ca.L[a] = h_L[a];
    ca.G[a] = h_G[a];
    ca.qout[a] = h_qout[a];
  }
  ca.cells = prod(h_L, d);
  ca.M = prod(h_G, d);
  ca.half = ca.cells / h_L[d - 1] * (h_L[d - 1] / 2 + 1);
  for (int p = 0; p < nprod; ++p)
    FLPR_CHECK_ARG(h_kidx[p] >= 0 && h_kidx[p] < nkern, "conv_full: kidx[%d]=%d", p, h_kidx[p]);
  if (ws_bytes < flpr_conv_ws(handle, d, h_L, nprod, prec)) {
    set_error("conv_full: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  const int B = conv_batch(d, h_L, nprod, prec);
  FLPR_CHECK_ARG((int64_t)B * ca.cells < ((int64_t)1 << 31),
                 "conv_full: grid too large for 32-bit batch indexing");
  const size_t es = prec == FLPR_PREC_F32 ? 4 : 8;
  Arena ar(d_ws, ws_bytes);
  char* pbuf = ar.take<char>((size_t)B * ca.half * 2 * es);
  char* rbuf = ar.take<char>((size_t)B * ca.cells * es);
  size_t work_bytes = ar.size - align_up(ar.used);
  char* work = ar.take<char>(1);
  cudaStream_t s = as_stream(stream);
  ProdBatch batch;
  const int ctype = prec == FLPR_PREC_F32 ? CUFFT_C2R : CUFFT_Z2D;
  for (int p0 = 0; p0 < nprod; p0 += B) {
    int nb = nprod - p0 < B ? nprod - p0 : B;
    for (int b = 0; b < nb; ++b) {
      ProdDesc pd{};
      pd.chan = h_chan[p0 + b];
      pd.hidx = h_kidx[p0 + b];
      batch.p[b] = pd;
    }
    int blocks = grid_blocks((int64_t)nb * ca.half);
    if (prec == FLPR_PREC_F32) {
      product_full_kernel<float><<<blocks, 256, 0, s>>>(ca, nb, batch, (const float2*)d_spec,
                                                        (const double2*)d_K, (float2*)pbuf);
    } else {
      product_full_kernel<double><<<blocks, 256, 0, s>>>(ca, nb, batch, (const double2*)d_spec,
                                                         (const double2*)d_K, (double2*)pbuf);
    }
    FLPR_LAUNCH_CHECK();
    FLPR_TRY(plans_of(handle).exec(grid_plan(d, h_L, ctype, nb), pbuf, rbuf, work, work_bytes, s));
    int cb = grid_blocks((int64_t)nb * ca.M);
    if (prec == FLPR_PREC_F32) {
      crop_kernel<float><<<cb, 256, 0, s>>>(ca, nb, p0, (const float*)rbuf, add_eps,
                                            (float*)d_out);
    } else {
      crop_kernel<double><<<cb, 256, 0, s>>>(ca, nb, p0, (const double*)rbuf, add_eps,
                                             (double*)d_out);
    }
    FLPR_LAUNCH_CHECK();
  }
  return FLPR_OK;
}

int flpr_oversample_crop(int d, const int* h_Lout, const int* h_Lin, int nchan,
                         const double* h_tau, int ratio, const void* d_in, void* d_out, int prec,
                         void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 3, "oversample_crop: d=%d", d);
  FLPR_CHECK_ARG(nchan >= 1 && ratio >= 1, "oversample_crop: nchan=%d ratio=%d", nchan, ratio);
  FLPR_CHECK_ARG(prec == FLPR_PREC_F32 || prec == FLPR_PREC_F64, "oversample_crop: precision");
  OverArgs a;
  memset(&a, 0, sizeof(a));
  a.d = d;
  a.C = nchan;
  double tprod = 1.0;
  a.half_o = 1;
  a.half_i = 1;
  for (int ax = 0; ax < d; ++ax) {
    FLPR_CHECK_ARG(h_Lout[ax] >= 1 && h_Lin[ax] >= h_Lout[ax], "oversample_crop: sizes");
    a.Lo[ax] = h_Lout[ax];
    a.Li[ax] = h_Lin[ax];
    a.tau[ax] = h_tau[ax];
    tprod *= h_tau[ax];
    a.half_o *= ax == d - 1 ? h_Lout[ax] / 2 + 1 : h_Lout[ax];
    a.half_i *= ax == d - 1 ? h_Lin[ax] / 2 + 1 : h_Lin[ax];
  }
  a.kn0 = sqrt(tprod / pow(M_PI, (double)d));
  a.inv_rd = 1.0 / pow((double)ratio, (double)d);
  const int64_t total = (int64_t)nchan * a.half_o;
  int nb = (int)((total + 255) / 256);
  if (nb > 16 * sm_count()) nb = 16 * sm_count();
  cudaStream_t s = as_stream(stream);
  if (prec == FLPR_PREC_F32)
    oversample_crop_kernel<float2><<<nb, 256, 0, s>>>(a, static_cast<const float2*>(d_in),
                                                      static_cast<float2*>(d_out));
  else
    oversample_crop_kernel<double2><<<nb, 256, 0, s>>>(a, static_cast<const double2*>(d_in),
                                                       static_cast<double2*>(d_out));
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
