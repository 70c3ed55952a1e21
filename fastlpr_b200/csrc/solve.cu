// Local polynomial solve at every (grid point, bandwidth).
#include "common.cuh"
#include "linalg.cuh"

namespace flpr {

constexpr int kMaxSolveChan = 64;
constexpr int kMaxDotChan = 32;

// Order-preserving map of a double onto an unsigned 64-bit integer.
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered(unsigned long long b) {
  b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
  return __longlong_as_double((long long)b);
}

// Largest value (absolute value with use_abs; NaN ignored) over the nt
// diagonal planes k of S (offset (k nt - k (k-1)/2) planes), as ordered bits
// atomically maxed into *out; vec: the planes start on 16-byte boundaries
// and hold whole vectors, so each load takes 16 bytes.
__device__ __forceinline__ void max_in(double v, int use_abs, unsigned long long& best) {
  if (use_abs) v = fabs(v);
  const unsigned long long b = ordered_bits(v);
  if (v == v && b > best) best = b;
}

template <typename Real>
__global__ void diag_max_kernel(int64_t plane_len, int nt, const Real* __restrict__ S, int use_abs,
                                int vec, unsigned long long* __restrict__ out) {
  __shared__ unsigned long long sh[256];
  unsigned long long best = ordered_bits(-INFINITY);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int k = 0; k < nt; ++k) {
    const Real* P = S + (int64_t)(k * nt - k * (k - 1) / 2) * plane_len;
    if (vec && sizeof(Real) == 4) {
      const float4* P4 = reinterpret_cast<const float4*>(P);
      for (int64_t i = t0; i < plane_len / 4; i += stride) {
        const float4 q = P4[i];
        max_in(q.x, use_abs, best);
        max_in(q.y, use_abs, best);
        max_in(q.z, use_abs, best);
        max_in(q.w, use_abs, best);
      }
    } else if (vec) {
      const double2* P2 = reinterpret_cast<const double2*>(P);
      for (int64_t i = t0; i < plane_len / 2; i += stride) {
        const double2 q = P2[i];
        max_in(q.x, use_abs, best);
        max_in(q.y, use_abs, best);
      }
    } else {
      for (int64_t i = t0; i < plane_len; i += stride) max_in((double)P[i], use_abs, best);
    }
  }
  sh[threadIdx.x] = best;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s && sh[threadIdx.x + s] > sh[threadIdx.x]) sh[threadIdx.x] = sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(out, sh[0]);
}

__global__ void bits_init_kernel(unsigned long long* bits) { bits[0] = ordered_bits(-INFINITY); }

__global__ void scalar_from_bits_kernel(const unsigned long long* bits, double factor, double* out) {
  out[0] = from_ordered(bits[0]) * factor;
}

// Solve vector z = (S + lam I)^-1 e1 at element t of the (H, M) planes, or
// 1/max(s, max(s) reg) for order 0.  Returns false if singular.
template <typename Real, int NT>
__device__ __forceinline__ bool zvec_at(int order, int64_t HM, int64_t t, const Real* __restrict__ S,
                                        double scal, double reg, double (&z)[NT]) {
  if (order == 0) {
    const double thr = scal * reg;
    const double s = (double)S[t];
    z[0] = 1.0 / (s > thr ? s : thr);
    return true;
  }
  constexpr int NS = NT * (NT + 1) / 2;
  double Ap[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) Ap[k] = (double)S[(int64_t)k * HM + t];
  return solve_e1_fixed<NT>(Ap, scal, z);
}

// Thread per (bandwidth, grid point) for the first HT bandwidths.
// S: (ns, H, M); T: (nt, C, HT, M); m: (HT, M, C) float64.
template <typename Real, int NT>
__global__ void solve_kernel(int order, int H, int HT, int64_t M, int C,
                             const Real* __restrict__ S, const Real* __restrict__ T, double reg,
                             const double* __restrict__ scalar, double* __restrict__ m) {
  const int64_t HM = (int64_t)H * M;
  const int64_t HTM = (int64_t)HT * M;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < HTM;
       t += (int64_t)gridDim.x * blockDim.x) {
    double z[NT];
    const bool ok = zvec_at<Real, NT>(order, HM, t, S, scalar[0], reg, z);
    double* mo = m + t * C;
    for (int c = 0; c < C; ++c) {
      double v = 0.0;
#pragma unroll
      for (int i = 0; i < NT; ++i) v += z[i] * (double)T[((int64_t)i * C + c) * HTM + t];
      mo[c] = ok ? v : NAN;
    }
  }
}

// Solve fused with the dual-form reductions.  blockIdx.y = bandwidth h < HT.
// Writes m for the first nkeep channels to mkeep (HT, M, nkeep) and adds
// dots[c][h] += sum_g m_c(g) Q[g][c] for every channel c < C.
template <typename Real, int NT>
__global__ void solve_reduce_kernel(int order, int H, int HT, int64_t M, int C,
                                    const Real* __restrict__ S, const Real* __restrict__ T,
                                    double reg, const double* __restrict__ scalar, int nkeep,
                                    double* __restrict__ mkeep, const double* __restrict__ Q,
                                    double* __restrict__ dots) {
  __shared__ double sh[32];
  const int h = blockIdx.y;
  const int64_t HM = (int64_t)H * M;
  const int64_t HTM = (int64_t)HT * M;
  double acc[kMaxDotChan];
#pragma unroll
  for (int c = 0; c < kMaxDotChan; ++c) acc[c] = 0.0;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < M;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = (int64_t)h * M + g;
    double z[NT];
    const bool ok = zvec_at<Real, NT>(order, HM, t, S, scalar[0], reg, z);
    const double* q = Q + g * C;
#pragma unroll
    for (int c = 0; c < kMaxDotChan; ++c) {
      if (c < C) {
        double v = 0.0;
#pragma unroll
        for (int i = 0; i < NT; ++i) v += z[i] * (double)T[((int64_t)i * C + c) * HTM + t];
        if (!ok) v = NAN;
        if (c < nkeep) mkeep[t * nkeep + c] = v;
        acc[c] += v * q[c];
      }
    }
  }
#pragma unroll
  for (int c = 0; c < kMaxDotChan; ++c) {
    if (c < C) {
      double v = acc[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      __syncthreads();
      if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += sh[w];
        atomicAdd(&dots[(int64_t)c * HT + h], sum);
      }
    }
  }
}

template <int NT>
static int launch_solve_reduce(int order, int H, int HT, int64_t M, int C, const void* d_S,
                               const void* d_T, double reg, const double* scalar, int nkeep,
                               double* mkeep, const double* Q, double* dots, int prec, dim3 grid,
                               cudaStream_t s) {
  if (prec == FLPR_PREC_F32) {
    solve_reduce_kernel<float, NT><<<grid, 256, 0, s>>>(order, H, HT, M, C, (const float*)d_S,
                                                        (const float*)d_T, reg, scalar, nkeep,
                                                        mkeep, Q, dots);
  } else {
    solve_reduce_kernel<double, NT><<<grid, 256, 0, s>>>(order, H, HT, M, C, (const double*)d_S,
                                                         (const double*)d_T, reg, scalar, nkeep,
                                                         mkeep, Q, dots);
  }
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int NT>
static int launch_solve(int order, int H, int HT, int64_t M, int C, const void* d_S,
                        const void* d_T, double reg, const double* scalar, double* m, int prec,
                        int nb, cudaStream_t s) {
  if (prec == FLPR_PREC_F32) {
    solve_kernel<float, NT><<<nb, 256, 0, s>>>(order, H, HT, M, C, (const float*)d_S,
                                               (const float*)d_T, reg, scalar, m);
  } else {
    solve_kernel<double, NT><<<nb, 256, 0, s>>>(order, H, HT, M, C, (const double*)d_S,
                                                (const double*)d_T, reg, scalar, m);
  }
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

static int blocks_for(int64_t total, int per_sm) {
  int64_t b = (total + 255) / 256;
  int64_t cap = (int64_t)per_sm * sm_count();
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

__global__ void scalar_max_kernel(double* __restrict__ scalar, const double* __restrict__ floor_) {
  const double a = scalar[0], b = floor_[0];
  scalar[0] = a > b ? a : b;
}

// *d_scalar = max(*d_scalar, *d_floor): the regularisation scalar over the
// union of two bandwidth groups (lambda grows with max |diag S|)
int scalar_floor(double* d_scalar, const double* d_floor, cudaStream_t s) {
  if (d_floor == nullptr) return FLPR_OK;
  scalar_max_kernel<<<1, 1, 0, s>>>(d_scalar, d_floor);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int global_scalar(int order, int nt, int H, int64_t M, const void* d_S, double* d_scalar,
                  int prec, cudaStream_t s) {
  unsigned long long* bits = reinterpret_cast<unsigned long long*>(d_scalar);
  bits_init_kernel<<<1, 1, 0, s>>>(bits);
  FLPR_LAUNCH_CHECK();
  const int64_t plane = (int64_t)H * M;
  // every diagonal element k (k nt - k (k-1)/2) in one launch
  const int nb = blocks_for(plane / 4 + 1, 16);
  const bool aligned = (reinterpret_cast<uintptr_t>(d_S) & 15) == 0;
  if (prec == FLPR_PREC_F32) {
    const int vec = aligned && plane % 4 == 0;
    diag_max_kernel<float><<<nb, 256, 0, s>>>(plane, nt, (const float*)d_S, order > 0, vec, bits);
  } else {
    const int vec = aligned && plane % 2 == 0;
    diag_max_kernel<double><<<nb, 256, 0, s>>>(plane, nt, (const double*)d_S, order > 0, vec,
                                               bits);
  }
  FLPR_LAUNCH_CHECK();
  scalar_from_bits_kernel<<<1, 1, 0, s>>>(bits, order > 0 ? 1e-6 : 1.0, d_scalar);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // namespace flpr

using namespace flpr;

extern "C" {

static int solve_reduce_impl(int order, int nt, int H, int HT, int64_t M, int C,
                             const void* d_S, const void* d_T, double reg, int nkeep,
                             double* d_mkeep, const double* d_Q, double* d_dots,
                             double* d_scalar, bool scalar_given, int prec, void* stream) {
  FLPR_CHECK_ARG(order >= 0 && order <= 2, "solve_reduce: order=%d", order);
  FLPR_CHECK_ARG(nt >= 1 && nt <= kMaxNt, "solve_reduce: nt=%d", nt);
  FLPR_CHECK_ARG(order > 0 || nt == 1, "solve_reduce: order 0 needs nt=1");
  FLPR_CHECK_ARG(H >= 1 && M >= 1 && C >= 1 && C <= kMaxDotChan, "solve_reduce: H=%d C=%d", H, C);
  FLPR_CHECK_ARG(HT >= 1 && HT <= H, "solve_reduce: HT=%d", HT);
  FLPR_CHECK_ARG(nkeep >= 0 && nkeep <= C, "solve_reduce: nkeep=%d", nkeep);
  cudaStream_t s = as_stream(stream);
  if (!scalar_given) FLPR_TRY(global_scalar(order, nt, H, M, d_S, d_scalar, prec, s));
  FLPR_CUDA(cudaMemsetAsync(d_dots, 0, sizeof(double) * (size_t)C * HT, s));
  int per_h = (blocks_for(M * HT, 4) + HT - 1) / HT;
  if (per_h < 2) per_h = 2;
  dim3 grid(per_h, HT);
  switch (nt) {
#define FLPR_NT(V)                                                                           \
  case V:                                                                                    \
    return launch_solve_reduce<V>(order, H, HT, M, C, d_S, d_T, reg, d_scalar, nkeep, d_mkeep, \
                                  d_Q, d_dots, prec, grid, s);
    FLPR_NT(1)
    FLPR_NT(2)
    FLPR_NT(3)
    FLPR_NT(4)
    FLPR_NT(6)
#undef FLPR_NT
    default:
      set_error("solve_reduce: nt=%d not supported", nt);
      return FLPR_ERR_ARG;
  }
}

int flpr_solve_reduce(int order, int nt, int H, int HT, int64_t M, int C, const void* d_S,
                      const void* d_T, double reg, int nkeep, double* d_mkeep, const double* d_Q,
                      double* d_dots, double* d_scalar, int prec, void* stream) {
  return solve_reduce_impl(order, nt, H, HT, M, C, d_S, d_T, reg, nkeep, d_mkeep, d_Q, d_dots,
                           d_scalar, false, prec, stream);
}

int flpr_solve_reduce_given(int order, int nt, int H, int HT, int64_t M, int C, const void* d_S,
                            const void* d_T, double reg, int nkeep, double* d_mkeep,
                            const double* d_Q, double* d_dots, const double* d_scalar, int prec,
                            void* stream) {
  FLPR_CHECK_ARG(d_scalar != nullptr, "solve_reduce_given: null scalar");
  return solve_reduce_impl(order, nt, H, HT, M, C, d_S, d_T, reg, nkeep, d_mkeep, d_Q, d_dots,
                           const_cast<double*>(d_scalar), true, prec, stream);
}

int flpr_scalar_of(int order, int nt, int H, int64_t M, const void* d_S, int prec,
                   const double* d_floor, double* d_scalar, void* stream) {
  FLPR_CHECK_ARG(order >= 0 && order <= 2 && nt >= 1 && nt <= kMaxNt, "scalar_of: order/nt");
  FLPR_CHECK_ARG(H >= 1 && M >= 1 && d_S && d_scalar, "scalar_of: H=%d", H);
  cudaStream_t s = as_stream(stream);
  FLPR_TRY(global_scalar(order, nt, H, M, d_S, d_scalar, prec, s));
  return scalar_floor(d_scalar, d_floor, s);
}

int flpr_solve(int order, int nt, int H, int HT, int64_t M, int C, const void* d_S,
               const void* d_T, double reg, double* d_m, double* d_scalar, int prec,
               void* stream) {
  FLPR_CHECK_ARG(order >= 0 && order <= 2, "solve: order=%d", order);
  FLPR_CHECK_ARG(nt >= 1 && nt <= kMaxNt, "solve: nt=%d", nt);
  FLPR_CHECK_ARG(order > 0 || nt == 1, "solve: order 0 needs nt=1");
  FLPR_CHECK_ARG(H >= 1 && M >= 1 && C >= 1 && C <= kMaxSolveChan, "solve: H=%d M=%lld C=%d", H,
                 (long long)M, C);
  FLPR_CHECK_ARG(HT >= 1 && HT <= H, "solve: HT=%d not in [1, H=%d]", HT, H);
  cudaStream_t s = as_stream(stream);
  // lambda = 1e-6 * max |diag S| (order >= 1, regression.py:243-267) or
  // max S (order 0, regression.py:207-212), over every bandwidth
  FLPR_TRY(global_scalar(order, nt, H, M, d_S, d_scalar, prec, s));
  int sb = blocks_for((int64_t)HT * M, 8);
  switch (nt) {
#define FLPR_NT(V)                                                                               \
  case V:                                                                                        \
    return launch_solve<V>(order, H, HT, M, C, d_S, d_T, reg, d_scalar, d_m, prec, sb, s);
    FLPR_NT(1)
    FLPR_NT(2)
    FLPR_NT(3)
    FLPR_NT(4)
    FLPR_NT(6)
#undef FLPR_NT
    default:
      set_error("solve: nt=%d not supported", nt);
      return FLPR_ERR_ARG;
  }
}

}  // extern "C"
