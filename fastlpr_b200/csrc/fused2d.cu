// Fused 2-D FP32 convolution + solve for the LPR GCV sweep.
//
// The Gaussian kernel spectrum is separable, K(w0, w1) = A0(w0) A1(w1), so
// the inverse transform of every product Y_c K splits into
//   column pass: W_{c,a0,h}(x0, w1) = IFFT_0(Y_c(., w1) A0_{h,a0})(x0), x0 cropped,
//   row pass:    r(x0, x1) = C2R_1(W(x0, .) A1_{h,a1})(x1), x1 cropped,
// and W is shared by every moment element with the same axis-0 exponent.
//
// Each 1-D transform of length N = 32 E is one warp (four-step form,
// N = E x 32): lane l holds x[32 s + l] in slot s; a radix-2 DIF over the E
// slots, a twiddle step, a transpose through a per-warp shared-memory
// buffer, and a second register DFT of length E leave lane t, slot s holding
// X[t % E + E (t / E + (32 / E) brev(s))].  Two real row products share one
// complex transform (both spectra are Hermitian).  The row pass of the T
// elements is fused with the per-point FP64 solve and the dual-form
// reductions, so neither the T planes nor the probe fits touch HBM.
#include "common.cuh"
#include "linalg.cuh"
#include "plans.cuh"

namespace flpr {

int global_scalar(int order, int nt, int H, int64_t M, const void* d_S, double* d_scalar, int prec,
                  cudaStream_t s);
int scalar_floor(double* d_scalar, const double* d_floor, cudaStream_t s);

namespace {

constexpr int kColWarps = 8;    // columns per column-pass CTA (one per warp)
constexpr int kRowWarps = 8;    // (row, job) items per S row-pass CTA (one per warp)
constexpr int kTWarps = 4;      // warps of a T row-pass CTA (8 products per round)
constexpr int kMaxSlots = 64;
constexpr int kMaxJobs = 64;
constexpr size_t kMaxSmem = 227 * 1024;
// Kernel factor entries below kBandEps of their peak are left out of both passes.
constexpr double kBandEps = 1e-11;
// The FP64 passes keep factor entries down to 1e-15 of their peak: the
// dropped share of any output stays below 1e-12.
constexpr double kBandEps64 = 1e-15;

// Complex sums on the packed two-lane FP32 instructions (add/sub.rn.f32x2):
// one instruction per complex add, each lane rounded as the scalar add.
__device__ __forceinline__ unsigned long long pack2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(d);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(d);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Complex vector type of a real type (float2 / double2).
template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using V = float2;
  __host__ __device__ static V make(float a, float b) { return make_float2(a, b); }
};
template <>
struct Vec2<double> {
  using V = double2;
  __host__ __device__ static V make(double a, double b) { return make_double2(a, b); }
};
template <typename V>
struct RealOf;
template <>
struct RealOf<float2> {
  using T = float;
};
template <>
struct RealOf<double2> {
  using T = double;
};
template <typename V>
__device__ __forceinline__ V vmake(typename RealOf<V>::T a, typename RealOf<V>::T b) {
  return Vec2<typename RealOf<V>::T>::make(a, b);
}

__host__ __device__ constexpr int brev(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r = (r << 1) | ((x >> i) & 1);
  return r;
}
__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

// Floats of one warp's transpose buffer: E rows of 33 (padded), rounded so
// that the column-pass write-out (8 warps' buffers read side by side as
// float2) hits distinct banks: stride = 4 (mod 32) words.
__host__ __device__ constexpr int warp_buf_stride(int E) { return ((33 * E + 31) / 32) * 32 + 4; }

// Doubles of one warp's buffer in the FP64 passes: E rows of 33 real parts
// (the transpose runs the real and the imaginary parts in turn) for
// E >= 16, E rows of 33 complex values for E <= 8 (whose second stage mixes
// the parts); rounded up to an even count (16-byte alignment of double2).
__host__ __device__ constexpr int warp_buf_stride64(int E) {
  return ((E >= 16 ? 33 * E : 66 * E) + 1) & ~1;
}

// Elements of type T of one warp's buffer.
template <typename T>
__host__ __device__ constexpr int buf_stride(int E) {
  return sizeof(T) == 4 ? warp_buf_stride(E) : warp_buf_stride64(E);
}

// Twiddle table of one axis, N + 32 entries: tw2[k1 * 32 + l] = exp(2 pi i l k1 / N)
// for k1 < E, then tw32[m] = exp(2 pi i m / 32).
__host__ __device__ constexpr int twiddle_entries(int N) { return N + 32; }

// a * exp(2 pi i m / 32), m known after unrolling: quarter turns are exact.
template <typename V>
__device__ __forceinline__ V rot32(V a, int m, const V* __restrict__ tw32) {
  m &= 31;
  if (m == 0) return a;
  if (m == 8) return vmake<V>(-a.y, a.x);
  if (m == 16) return vmake<V>(-a.x, -a.y);
  if (m == 24) return vmake<V>(a.y, -a.x);
  return cmul(a, tw32[m]);
}

// In-register radix-2 DIF (inverse sign) over the E slots: slot s ends up
// holding output brev(s).  E <= 32, so every twiddle is a power of W_32.
template <int E, typename V>
__device__ __forceinline__ void dif_slots(V (&v)[E], const V* __restrict__ tw32) {
#pragma unroll
  for (int span = E / 2; span >= 1; span >>= 1) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      if ((s & span) == 0) {
        const V a = v[s], b = v[s + span];
        v[s] = cadd(a, b);
        v[s + span] = rot32(csub(a, b), (s & (span - 1)) * (16 / span), tw32);
      }
    }
  }
}

// Output index held by lane t, slot s after warp_ifft<E>.
template <int E>
__device__ __forceinline__ int out_index(int lane, int s) {
  constexpr int EB = ilog2(E);
  constexpr int P = 32 / E;
  return (lane & (E - 1)) + E * ((lane >> EB) + P * brev(s, EB));
}

// Inverse (unnormalised) FFT of length N = 32 E held by one warp.  On entry
// lane l, slot s holds x[32 s + l]; on exit lane t, slot s holds
// X[out_index<E>(t, s)].  buf: this warp's warp_buf_stride(E) floats, free
// again when the function returns.
template <int E>
__device__ __forceinline__ void warp_ifft(float2 (&v)[E], const float2* __restrict__ tw2,
                                          const float2* __restrict__ tw32, float* buf, int lane) {
  constexpr int EB = ilog2(E);
  constexpr int P = 32 / E;
  // DFT over n1 (n = 32 n1 + n2) for each n2 = lane
  dif_slots<E>(v, tw32);
  // twiddle W_N^(n2 k1), k1 = brev(s)
#pragma unroll
  for (int s = 1; s < E; ++s) v[s] = cmul(v[s], tw2[brev(s, EB) * 32 + lane]);
  // transpose: lane t gathers row k1 = t % E (all 32 n2), real and imaginary
  // parts in turn through the same E x 33 buffer
  const int k1 = lane & (E - 1), part = lane >> EB;
  float ur[32], ui[32];
#pragma unroll
  for (int s = 0; s < E; ++s) buf[brev(s, EB) * 33 + lane] = v[s].x;
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 32; ++j) ur[j] = buf[k1 * 33 + j];
  __syncwarp();
#pragma unroll
  for (int s = 0; s < E; ++s) buf[brev(s, EB) * 33 + lane] = v[s].y;
  __syncwarp();
#pragma unroll
  for (int j = 0; j < 32; ++j) ui[j] = buf[k1 * 33 + j];
  __syncwarp();
  // 32-point DFT over n2 at k2 = part + P k2': n2 = n2' + E q; the q-sum is a
  // P-point DFT at frequency `part`, then W_32^(n2' part), then a length-E
  // DFT over n2'
#pragma unroll
  for (int n = 0; n < E; ++n) {
    float2 z = make_float2(ur[n], ui[n]);
    if constexpr (P > 1) {
#pragma unroll
      for (int q = 1; q < P; ++q)
        z = cadd(z, cmul(make_float2(ur[n + E * q], ui[n + E * q]), tw32[(E * q * part) & 31]));
      if (n > 0) z = cmul(z, tw32[(n * part) & 31]);
    }
    v[n] = z;
  }
  dif_slots<E>(v, tw32);
}

// warp_ifft in FP64 (same input and output layout).  The 32 values a lane
// gathers in the transpose would take 128 registers as doubles, so its
// second stage reads them from the buffer as it combines them: for E >= 16
// the P-point DFT (P <= 2) has real weights +-1 and the real and imaginary
// parts pass through a buffer of E x 33 doubles in turn, each overwriting
// the register it replaces; for E <= 8 the whole complex row goes through a
// buffer of E x 33 double2.  buf: this warp's warp_buf_stride64(E) doubles.
template <int E>
__device__ __forceinline__ void warp_ifft64(double2 (&v)[E], const double2* __restrict__ tw2,
                                            const double2* __restrict__ tw32, double* buf,
                                            int lane) {
  constexpr int EB = ilog2(E);
  constexpr int P = 32 / E;
  dif_slots<E>(v, tw32);
#pragma unroll
  for (int s = 1; s < E; ++s) v[s] = cmul(v[s], tw2[brev(s, EB) * 32 + lane]);
  const int k1 = lane & (E - 1), part = lane >> EB;
  if constexpr (P <= 2) {
    const double sgn = (P == 2 && part) ? -1.0 : 1.0;
#pragma unroll
    for (int s = 0; s < E; ++s) buf[brev(s, EB) * 33 + lane] = v[s].x;
    __syncwarp();
#pragma unroll
    for (int n = 0; n < E; ++n) {
      double z = buf[k1 * 33 + n];
      if constexpr (P == 2) z += sgn * buf[k1 * 33 + n + E];
      v[n].x = z;
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < E; ++s) buf[brev(s, EB) * 33 + lane] = v[s].y;
    __syncwarp();
#pragma unroll
    for (int n = 0; n < E; ++n) {
      double z = buf[k1 * 33 + n];
      if constexpr (P == 2) z += sgn * buf[k1 * 33 + n + E];
      v[n].y = z;
    }
    __syncwarp();
    if constexpr (P == 2) {
#pragma unroll
      for (int n = 1; n < E; ++n) v[n] = cmul(v[n], tw32[(n * part) & 31]);
    }
  } else {
    double2* cb = reinterpret_cast<double2*>(buf);
#pragma unroll
    for (int s = 0; s < E; ++s) cb[brev(s, EB) * 33 + lane] = v[s];
    __syncwarp();
#pragma unroll
    for (int n = 0; n < E; ++n) {
      double2 z = cb[k1 * 33 + n];
#pragma unroll
      for (int q = 1; q < P; ++q) z = cadd(z, cmul(cb[k1 * 33 + n + E * q], tw32[(E * q * part) & 31]));
      if (n > 0) z = cmul(z, tw32[(n * part) & 31]);
      v[n] = z;
    }
    __syncwarp();
  }
  dif_slots<E>(v, tw32);
}

// The inverse transform of the precision's vector type.
template <int E>
__device__ __forceinline__ void warp_ifft_t(float2 (&v)[E], const float2* tw2, const float2* tw32,
                                            float* buf, int lane) {
  warp_ifft<E>(v, tw2, tw32, buf, lane);
}
template <int E>
__device__ __forceinline__ void warp_ifft_t(double2 (&v)[E], const double2* tw2,
                                            const double2* tw32, double* buf, int lane) {
  warp_ifft64<E>(v, tw2, tw32, buf, lane);
}

// Twiddle tables of one axis (layout of twiddle_entries).
template <typename V>
__global__ void twiddle_table_kernel(int N, V* __restrict__ tab) {
  const int total = twiddle_entries(N);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    double sn, cs;
    if (k < N) {
      const int k1 = k / 32, l = k % 32;  // l * k1 < N
      sincospi(2.0 * (double)(l * k1) / (double)N, &sn, &cs);
    } else {
      sincospi(2.0 * (double)(k - N) / 32.0, &sn, &cs);
    }
    tab[k] = vmake<V>((typename RealOf<V>::T)cs, (typename RealOf<V>::T)sn);
  }
}

// Per-axis kernel factor spectra in the pass precision: F (H, npow, L0) for
// axis 0 (times `scale`) followed by (H, npow, L1) for axis 1.
template <typename V>
__global__ void factor_kernel(int64_t n0, int64_t ntot, double scale,
                              const double2* __restrict__ F, V* __restrict__ Ff) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ntot;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 f = F[i];
    const double s = i < n0 ? scale : 1.0;
    Ff[i] = vmake<V>((typename RealOf<V>::T)(f.x * s), (typename RealOf<V>::T)(f.y * s));
  }
}

// Band limit of the kernel factor spectra: kcut[axis * H + h] is the largest
// frequency index m <= N/2 (entries k and N - k) at which some power a has
// |F[h][a][.]| >= eps * max_k |F[h][a][k]|.  Both passes treat the terms
// beyond it as zero: their share of any output is below eps * N relative.
// grid (H, 2), one block per (bandwidth, axis).
__global__ void band_limit_kernel(int H, int npow, int L0, int L1, const double2* __restrict__ F,
                                  double eps, int* __restrict__ kcut) {
  __shared__ double smax[32];
  __shared__ int scut[32];
  const int h = blockIdx.x, ax = blockIdx.y;
  const int N = ax == 0 ? L0 : L1;
  const double2* base = F + (ax == 0 ? 0 : (size_t)H * npow * L0) + (size_t)h * npow * N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  int best = 0;
  for (int a = 0; a < npow; ++a) {
    const double2* f = base + (size_t)a * N;
    double m = 0.0;
    for (int k = threadIdx.x; k < N; k += blockDim.x) m = fmax(m, f[k].x * f[k].x + f[k].y * f[k].y);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) smax[warp] = m;
    __syncthreads();
    double mx = 0.0;
    for (int w = 0; w < nw; ++w) mx = fmax(mx, smax[w]);
    const double thr = eps * eps * mx;
    int kc = 0;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      const double v = f[k].x * f[k].x + f[k].y * f[k].y;
      if (mx > 0.0 && v >= thr) kc = max(kc, min(k, N - k));
    }
    for (int o = 16; o > 0; o >>= 1) kc = max(kc, __shfl_xor_sync(0xffffffffu, kc, o));
    if (lane == 0) scut[warp] = kc;
    __syncthreads();
    for (int w = 0; w < nw; ++w) best = max(best, scut[w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) kcut[ax * H + h] = best;
}

template <int E, typename V>
__device__ __forceinline__ void load_twiddles(V* s_tab, const V* __restrict__ tab) {
  constexpr int T = twiddle_entries(32 * E);
  for (int i = threadIdx.x; i < T; i += blockDim.x) s_tab[i] = tab[i];
}

// (C, L0, L1h) -> (C, L1h, L0)
template <typename V>
__global__ void transpose_spec_kernel(int C, int L0, int L1h, const V* __restrict__ in,
                                      V* __restrict__ out) {
  __shared__ V tile[32][33];
  const int c = blockIdx.z;
  const int w0 = blockIdx.y * 32, w1 = blockIdx.x * 32;
  const V* src = in + (size_t)c * L0 * L1h;
  V* dst = out + (size_t)c * L0 * L1h;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int r = w0 + i, col = w1 + threadIdx.x;
    if (r < L0 && col < L1h) tile[i][threadIdx.x] = src[(size_t)r * L1h + col];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int col = w1 + i, r = w0 + threadIdx.x;
    if (r < L0 && col < L1h) dst[(size_t)col * L0 + r] = tile[threadIdx.x][i];
  }
}

struct ColArgs {
  int L0, L1h, G0, q0;
  int npow, hbase, nslots;
  int slot_chan[kMaxSlots];
  int slot_pow[kMaxSlots];
};

// grid (ceil(L1h/8), nslots, Hc); warp w handles column blockIdx.x*8+w.
// W layout: [slot][hz][r][w1], r = x0 - q0 in [0, G0).  Each warp stages its
// cropped column in its own transpose buffer; the CTA then writes 8-column
// row segments.
template <int E, typename T>
__global__ void __launch_bounds__(kColWarps * 32, sizeof(T) == 4 ? (E <= 16 ? 3 : 2) : (E <= 16 ? 2 : 1))
colpass_kernel(ColArgs ca, const typename Vec2<T>::V* __restrict__ Yt,
               const typename Vec2<T>::V* __restrict__ F0f,
               const typename Vec2<T>::V* __restrict__ tab, const int* __restrict__ kcut1,
               typename Vec2<T>::V* __restrict__ W) {
  using V = typename Vec2<T>::V;
  constexpr int N = 32 * E;
  constexpr int SW = buf_stride<T>(E);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // columns beyond the axis-1 band limit are never read by the row pass
  const int kc1 = kcut1[ca.hbase + blockIdx.z];
  if (blockIdx.x * kColWarps > kc1) return;
  V* s_tw2 = reinterpret_cast<V*>(smem_raw);
  V* s_tw32 = s_tw2 + N;
  T* bufs = reinterpret_cast<T*>(s_tw2 + twiddle_entries(N));
  load_twiddles<E>(s_tw2, tab);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = blockIdx.y, hz = blockIdx.z, h = ca.hbase + hz;
  const int c = ca.slot_chan[slot], a0 = ca.slot_pow[slot];
  const int w1 = blockIdx.x * kColWarps + warp;
  T* buf = bufs + warp * SW;
  if (w1 < ca.L1h && w1 <= kc1) {
    const V* col = Yt + ((size_t)c * ca.L1h + w1) * N + lane;
    const V* f = F0f + ((size_t)h * ca.npow + a0) * N + lane;
    V v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) v[s] = cmul(col[32 * s], f[32 * s]);
    warp_ifft_t<E>(v, s_tw2, s_tw32, buf, lane);
    V* stage = reinterpret_cast<V*>(buf);
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int r = out_index<E>(lane, s) - ca.q0;
      if (r >= 0 && r < ca.G0) stage[r] = v[s];
    }
  }
  __syncthreads();
  V* out = W + ((size_t)slot * gridDim.z + hz) * ca.G0 * ca.L1h;
  for (int i = threadIdx.x; i < ca.G0 * kColWarps; i += blockDim.x) {
    const int r = i / kColWarps, wl = i - r * kColWarps;
    const int colw = blockIdx.x * kColWarps + wl;
    if (colw < ca.L1h && colw <= kc1)
      out[(size_t)r * ca.L1h + colw] = reinterpret_cast<const V*>(bufs + wl * SW)[r];
  }
}

// Solve vectors z = (S + lam I)^-1 e1 per (bandwidth, grid point); order 0
// stores 1/max(s, max(s) reg).  S: (ns, H, M) float or double; z: (H, M, NT)
// double.
template <int NT, typename TS>
__global__ void zvec_kernel(int order, int H, int64_t M, const TS* __restrict__ S,
                            const double* __restrict__ scalar, double reg, double* __restrict__ z) {
  constexpr int NS = NT * (NT + 1) / 2;
  const int64_t HM = (int64_t)H * M;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < HM;
       t += (int64_t)gridDim.x * blockDim.x) {
    double zz[NT];
    if (order == 0) {
      const double thr = scalar[0] * reg;
      const double s = (double)S[t];
      zz[0] = 1.0 / (s > thr ? s : thr);
    } else {
      double Ap[NS];
#pragma unroll
      for (int k = 0; k < NS; ++k) Ap[k] = (double)S[(int64_t)k * HM + t];
      if (!solve_e1_fixed<NT>(Ap, scalar[0], zz)) {
#pragma unroll
        for (int i = 0; i < NT; ++i) zz[i] = NAN;
      }
    }
#pragma unroll
    for (int i = 0; i < NT; ++i) z[t * NT + i] = zz[i];
  }
}

struct RowJob {
  short slot_a, pow_a, out_a;
  short slot_b, pow_b, out_b;  // slot_b < 0: single product
};

struct RowArgs {
  int L1, L1h, G0, G1, q1;
  int npow, hbase;
  int njobs;
  RowJob jobs[kMaxJobs];
};

// Slot s of the Hermitian extension of the product W_row * A1: element
// k = 32 s + lane, mirrored (conjugated) above N/2; the DC and Nyquist terms
// are real; frequencies beyond the band limit kc are zero.
// lo = row + lane, hi = row + N - lane.
template <int E, typename V>
__device__ __forceinline__ V herm_product(const V* __restrict__ wlo, const V* __restrict__ flo,
                                          const V* __restrict__ whi, const V* __restrict__ fhi,
                                          int s, int lane, int kc) {
  constexpr int N = 32 * E;
  V p = vmake<V>(0, 0);
  if (s < E / 2) {
    if (32 * s + lane <= kc) p = cmul(wlo[32 * s], flo[32 * s]);
    if (s == 0 && lane == 0) p.y = 0.0f;
  } else {
    if (N - 32 * s - lane <= kc) p = cmul(whi[-32 * s], fhi[-32 * s]);
    p.y = (s == E / 2 && lane == 0) ? 0.0f : -p.y;
  }
  return p;
}

// One warp: the inverse transform of job jb for row r; on return lane t,
// slot s holds the products a (real part) and b (imaginary part) at
// x1 = out_index(t, s).
template <int E, typename T>
__device__ __forceinline__ void row_fft(const RowArgs& ra, const RowJob& jb, int r, int hz, int h,
                                        int nslots_w, const typename Vec2<T>::V* __restrict__ W,
                                        const typename Vec2<T>::V* __restrict__ F1f,
                                        const typename Vec2<T>::V* s_tw2,
                                        const typename Vec2<T>::V* s_tw32, T* buf, int lane,
                                        int kc, typename Vec2<T>::V (&v)[E]) {
  using V = typename Vec2<T>::V;
  constexpr int N = 32 * E;
  const size_t rowstride = (size_t)ra.L1h;
  const V* wa = W + (((size_t)jb.slot_a * nslots_w + hz) * ra.G0 + r) * rowstride;
  const V* fa = F1f + ((size_t)h * ra.npow + jb.pow_a) * N;
  if (jb.slot_b >= 0) {
    const V* wb = W + (((size_t)jb.slot_b * nslots_w + hz) * ra.G0 + r) * rowstride;
    const V* fb = F1f + ((size_t)h * ra.npow + jb.pow_b) * N;
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const V pa =
          herm_product<E>(wa + lane, fa + lane, wa + N - lane, fa + N - lane, s, lane, kc);
      const V pb =
          herm_product<E>(wb + lane, fb + lane, wb + N - lane, fb + N - lane, s, lane, kc);
      v[s] = vmake<V>(pa.x - pb.y, pa.y + pb.x);
    }
  } else {
#pragma unroll
    for (int s = 0; s < E; ++s)
      v[s] = herm_product<E>(wa + lane, fa + lane, wa + N - lane, fa + N - lane, s, lane, kc);
  }
  warp_ifft_t<E>(v, s_tw2, s_tw32, buf, lane);
}

// S pass: grid (ceil(G0 * njobs / 8), Hc); warp w takes item blockIdx.x*8+w =
// (row, job).  S planes (ns, H, G0*G1) in the pass precision, written
// straight from the registers (consecutive lanes hold consecutive x1).
template <int E, typename T>
__global__ void __launch_bounds__(kRowWarps * 32, sizeof(T) == 4 ? (E <= 16 ? 3 : 2) : (E <= 16 ? 2 : 1))
rowpass_s_kernel(RowArgs ra, int H, int nslots_w, const typename Vec2<T>::V* __restrict__ W,
                 const typename Vec2<T>::V* __restrict__ F1f,
                 const typename Vec2<T>::V* __restrict__ tab, const int* __restrict__ kcut1,
                 T* __restrict__ S) {
  using V = typename Vec2<T>::V;
  constexpr int N = 32 * E;
  constexpr int SW = buf_stride<T>(E);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* s_tw2 = reinterpret_cast<V*>(smem_raw);
  V* s_tw32 = s_tw2 + N;
  T* bufs = reinterpret_cast<T*>(s_tw2 + twiddle_entries(N));
  load_twiddles<E>(s_tw2, tab);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * kRowWarps + warp;
  if (item >= ra.G0 * ra.njobs) return;
  const int r = item / ra.njobs, j = item - r * ra.njobs;
  const int hz = blockIdx.y, h = ra.hbase + hz;
  const int64_t M = (int64_t)ra.G0 * ra.G1;
  const RowJob jb = ra.jobs[j];
  const bool pair = jb.slot_b >= 0;
  V v[E];
  row_fft<E, T>(ra, jb, r, hz, h, nslots_w, W, F1f, s_tw2, s_tw32, bufs + warp * SW, lane,
                kcut1[h], v);
  T* da = S + ((size_t)jb.out_a * H + h) * M + (size_t)r * ra.G1;
  T* db = S + ((size_t)(pair ? jb.out_b : jb.out_a) * H + h) * M + (size_t)r * ra.G1;
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int x = out_index<E>(lane, s) - ra.q1;
    if (x >= 0 && x < ra.G1) {
      da[x] = v[s].x;
      if (pair) db[x] = v[s].y;
    }
  }
}

// Shared memory of the T pass: twiddles and two transpose buffers per warp
// (rounds alternate between them; a warp's job leaves its two cropped
// products there).
template <typename T>
inline size_t t_smem_bytes(int E, int nwarps, int njobs, int G1) {
  (void)njobs;
  (void)G1;
  return 2 * sizeof(T) * (size_t)twiddle_entries(32 * E) +
         sizeof(T) * (size_t)2 * nwarps * buf_stride<T>(E);
}

// Warps of a T-pass CTA: rounds of kTWarps jobs, or one round when there
// are fewer jobs.  Four warps at the 112-register cap let four CTAs share
// an SM (16 warps; six-warp CTAs are allocated as eight warps, two CTAs).
inline int t_warps(int njobs) { return njobs < kTWarps ? njobs : kTWarps; }

// T pass fused with the solve and the dual-form reductions: grid (Hc, G0),
// t_warps(njobs) warps.  Product p = c * NT + i is half p % 2 of job p / 2.
// In round k the warps compute jobs k * nwarps + w, each leaving its two
// cropped products in its buffer of parity k % 2; then, for the channels
// completed in that round, m_c(x1) = sum_i z_i(x1) T(p, x1) with z the row's
// solve vectors, the response fits go to `my`, and sum_x1 m_c Q_c
// accumulates into one partial per (c, h, row).  A channel's NT products
// span at most two consecutive rounds (NT <= 2 nwarps + 1), so the buffers
// of the previous round still hold its earlier products.
template <int E, int NT, typename T>
__device__ __forceinline__ void rowpass_t_solve_body(
    RowArgs ra, int H, int nslots_w, const typename Vec2<T>::V* __restrict__ W,
    const typename Vec2<T>::V* __restrict__ F1f, const typename Vec2<T>::V* __restrict__ tab,
    const int* __restrict__ kcut1, int C, int ny, const double* __restrict__ zg,
    const double* __restrict__ Q, double* __restrict__ my, double* __restrict__ dpart) {
  using V = typename Vec2<T>::V;
  constexpr int N = 32 * E;
  constexpr int SW = buf_stride<T>(E);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[kTWarps * 32];
  V* s_tw2 = reinterpret_cast<V*>(smem_raw);
  V* s_tw32 = s_tw2 + N;
  T* bufs = reinterpret_cast<T*>(s_tw2 + twiddle_entries(N));
  const int nwarps = blockDim.x >> 5;
  // bandwidth fastest: the CTAs of one row (sharing its deposits Q) run together
  const int hz = blockIdx.x, r = blockIdx.y, h = ra.hbase + hz;
  const int64_t M = (int64_t)ra.G0 * ra.G1;
  const int G1 = ra.G1, njobs = ra.njobs;
  {
    // start every W row this row's jobs read (up to the band limit) and the
    // row's solve vectors on their way into L2 before the first transform
    const int lines = ((kcut1[h] + 1) * (int)sizeof(V) + 127) / 128;
    const int per_job = 2 * lines;
    for (int t = threadIdx.x; t < njobs * per_job; t += blockDim.x) {
      const int j = t / per_job, rem = t - j * per_job;
      const int side = rem / lines, l = rem - side * lines;
      const int slot = side == 0 ? ra.jobs[j].slot_a : ra.jobs[j].slot_b;
      if (slot < 0) continue;
      const char* row = reinterpret_cast<const char*>(
          W + (((size_t)slot * nslots_w + hz) * ra.G0 + r) * (size_t)ra.L1h);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(row + 128 * l));
    }
    const char* zr = reinterpret_cast<const char*>(zg + ((int64_t)h * M + (int64_t)r * G1) * NT);
    const int zl = (G1 * NT * (int)sizeof(double) + 127) / 128;
    for (int l = threadIdx.x; l < zl; l += blockDim.x)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(zr + 128 * l));
  }
  load_twiddles<E>(s_tw2, tab);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kc = kcut1[h];
  const int nprod = C * NT;
  for (int r0 = 0; r0 < njobs; r0 += nwarps) {
    const int j = r0 + warp;
    T* buf = bufs + ((size_t)(((r0 / nwarps) & 1) * nwarps) + warp) * SW;
    if (j < njobs) {
      const RowJob jb = ra.jobs[j];
      const bool pair = jb.slot_b >= 0;
      V v[E];
      row_fft<E, T>(ra, jb, r, hz, h, nslots_w, W, F1f, s_tw2, s_tw32, buf, lane, kc, v);
#pragma unroll
      for (int s = 0; s < E; ++s) {
        const int x = out_index<E>(lane, s) - ra.q1;
        if (x >= 0 && x < G1) {
          buf[x] = v[s].x;
          if (pair) buf[G1 + x] = v[s].y;
        }
      }
    }
    __syncthreads();
    // channels whose NT products all came out of this round
    const int p_end = min(nprod, 2 * (r0 + nwarps));
    const int c_begin = (2 * r0) / NT, c_end = p_end / NT;
    for (int c = c_begin; c < c_end; ++c) {
      const T* src[NT];
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        const int p = c * NT + i, jj = p >> 1, kk = jj / nwarps;
        src[i] = bufs + ((size_t)((kk & 1) * nwarps) + (jj - kk * nwarps)) * SW + (p & 1) * G1;
      }
      double acc = 0.0;
      for (int x = threadIdx.x; x < G1; x += blockDim.x) {
        const int64_t g = (int64_t)r * G1 + x;
        const double* z = zg + ((int64_t)h * M + g) * NT;
        double m = 0.0;
#pragma unroll
        for (int i = 0; i < NT; ++i) m += z[i] * (double)src[i][x];
        if (c < ny) my[((int64_t)h * M + g) * ny + c] = m;
        acc += m * Q[g * C + c];
      }
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) red[c * nwarps + warp] = acc;  // C * nwarps <= 32 * kTWarps
    }
    __syncthreads();  // the next round overwrites the buffers
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nwarps; ++w) s += red[c * nwarps + w];
    dpart[((int64_t)c * H + h) * ra.G0 + r] = s;
  }
}

// FP32: four CTAs of four warps per SM at the 112-register cap.
template <int E, int NT>
__global__ void __maxnreg__(E <= 16 ? 80 : 112)
rowpass_t_solve_kernel(RowArgs ra, int H, int nslots_w, const float2* __restrict__ W,
                       const float2* __restrict__ F1f, const float2* __restrict__ tab,
                       const int* __restrict__ kcut1, int C, int ny, const double* __restrict__ zg,
                       const double* __restrict__ Q, double* __restrict__ my,
                       double* __restrict__ dpart) {
  rowpass_t_solve_body<E, NT, float>(ra, H, nslots_w, W, F1f, tab, kcut1, C, ny, zg, Q, my,
                                     dpart);
}

// FP64: the 32-slot transform alone holds 128 registers; two CTAs per SM.
template <int E, int NT>
__global__ void __launch_bounds__(kTWarps * 32, E <= 16 ? 4 : 2)
rowpass_t_solve64_kernel(RowArgs ra, int H, int nslots_w, const double2* __restrict__ W,
                         const double2* __restrict__ F1f, const double2* __restrict__ tab,
                         const int* __restrict__ kcut1, int C, int ny,
                         const double* __restrict__ zg, const double* __restrict__ Q,
                         double* __restrict__ my, double* __restrict__ dpart) {
  rowpass_t_solve_body<E, NT, double>(ra, H, nslots_w, W, F1f, tab, kcut1, C, ny, zg, Q, my,
                                      dpart);
}

// dots[c, h] = sum of the row partials (fixed order: deterministic).
__global__ void dots_reduce_kernel(int CH, int G0, const double* __restrict__ dpart,
                                   double* __restrict__ dots) {
  const int ch = blockIdx.x;
  __shared__ double sh[256];
  double s = 0.0;
  for (int r = threadIdx.x; r < G0; r += blockDim.x) s += dpart[(int64_t)ch * G0 + r];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0 && ch < CH) dots[ch] = sh[0];
}

}  // namespace

namespace {

template <typename K>
static int set_smem(K kernel, size_t bytes, int threads) {
  // the FFT passes re-read their kernel factor rows from L1: give shared
  // memory only what the resident CTAs use
  FLPR_CUDA(fit_carveout(kernel, threads, bytes));
  return FLPR_OK;
}

template <typename T>
static size_t warp_pass_smem(int E, int nwarps) {
  return 2 * sizeof(T) * (size_t)twiddle_entries(32 * E) +
         sizeof(T) * (size_t)nwarps * buf_stride<T>(E);
}

template <int E, typename T>
static int launch_col(const ColArgs& ca, int ncolblk, int nslots, int Hc,
                      const typename Vec2<T>::V* Yt, const typename Vec2<T>::V* F0f,
                      const typename Vec2<T>::V* tab, const int* kcut1, typename Vec2<T>::V* W,
                      cudaStream_t s) {
  const size_t smem = warp_pass_smem<T>(E, kColWarps);
  FLPR_TRY(set_smem(colpass_kernel<E, T>, smem, kColWarps * 32));
  colpass_kernel<E, T><<<dim3(ncolblk, nslots, Hc), kColWarps * 32, smem, s>>>(ca, Yt, F0f, tab,
                                                                             kcut1, W);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int E, typename T>
static int launch_row_s(const RowArgs& ra, int Hc, int H, int nslots_w,
                        const typename Vec2<T>::V* W, const typename Vec2<T>::V* F1f,
                        const typename Vec2<T>::V* tab, const int* kcut1, T* S, cudaStream_t s) {
  const size_t smem = warp_pass_smem<T>(E, kRowWarps);
  FLPR_TRY(set_smem(rowpass_s_kernel<E, T>, smem, kRowWarps * 32));
  const int items = ra.G0 * ra.njobs;
  rowpass_s_kernel<E, T><<<dim3((items + kRowWarps - 1) / kRowWarps, Hc), kRowWarps * 32, smem,
                           s>>>(ra, H, nslots_w, W, F1f, tab, kcut1, S);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int E, int NT>
static int launch_row_t_k(const RowArgs& ra, int Hc, int H, int nslots_w, const float2* W,
                          const float2* F1f, const float2* tab, const int* kcut1, int C, int ny,
                          const double* z, const double* Q, double* my, double* dpart,
                          cudaStream_t s) {
  const int nwarps = t_warps(ra.njobs);
  const size_t smem = t_smem_bytes<float>(E, nwarps, ra.njobs, ra.G1);
  FLPR_TRY(set_smem(rowpass_t_solve_kernel<E, NT>, smem, nwarps * 32));
  rowpass_t_solve_kernel<E, NT><<<dim3(Hc, ra.G0), nwarps * 32, smem, s>>>(
      ra, H, nslots_w, W, F1f, tab, kcut1, C, ny, z, Q, my, dpart);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}
template <int E, int NT>
static int launch_row_t_k(const RowArgs& ra, int Hc, int H, int nslots_w, const double2* W,
                          const double2* F1f, const double2* tab, const int* kcut1, int C, int ny,
                          const double* z, const double* Q, double* my, double* dpart,
                          cudaStream_t s) {
  const int nwarps = t_warps(ra.njobs);
  const size_t smem = t_smem_bytes<double>(E, nwarps, ra.njobs, ra.G1);
  FLPR_TRY(set_smem(rowpass_t_solve64_kernel<E, NT>, smem, nwarps * 32));
  rowpass_t_solve64_kernel<E, NT><<<dim3(Hc, ra.G0), nwarps * 32, smem, s>>>(
      ra, H, nslots_w, W, F1f, tab, kcut1, C, ny, z, Q, my, dpart);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int E, typename V>
static int launch_row_t(int nt, const RowArgs& ra, int Hc, int H, int nslots_w, const V* W,
                        const V* F1f, const V* tab, const int* kc, int C, int ny,
                        const double* z, const double* Q, double* my, double* dp, cudaStream_t s) {
  switch (nt) {
    case 1: return launch_row_t_k<E, 1>(ra, Hc, H, nslots_w, W, F1f, tab, kc, C, ny, z, Q, my, dp, s);
    case 3: return launch_row_t_k<E, 3>(ra, Hc, H, nslots_w, W, F1f, tab, kc, C, ny, z, Q, my, dp, s);
    case 6: return launch_row_t_k<E, 6>(ra, Hc, H, nslots_w, W, F1f, tab, kc, C, ny, z, Q, my, dp, s);
    default: set_error("fused2d: nt=%d", nt); return FLPR_ERR_ARG;
  }
}

// Slot/job tables of one configuration.
struct FusedTables {
  int nt, ns;
  int s_nslots, t_nslots;
  ColArgs s_col, t_col;
  RowArgs s_row, t_row;
  // S elements whose exponent an earlier element has (order 2: 6 of 21):
  // the S pass computes each exponent once, then copies dup_src -> dup_dst
  int ndup;
  int dup_src[55], dup_dst[55];
};

static void design_powers2(int order, int pw[][2], int* nt) {
  int k = 0;
  for (int tot = 0; tot <= order; ++tot)
    for (int px = tot; px >= 0; --px) {
      pw[k][0] = px;
      pw[k][1] = tot - px;
      ++k;
    }
  *nt = k;
}

static int build_tables(int order, int C, FusedTables* t) {
  int pw[10][2];
  int nt = 0;
  design_powers2(order, pw, &nt);
  if (order == 0) nt = 1;
  t->nt = nt;
  t->ns = nt * (nt + 1) / 2;
  // S elements (column-major lower triangle): exponent pw_i + pw_j
  int ep[55][2];
  int k = 0;
  for (int j = 0; j < nt; ++j)
    for (int i = j; i < nt; ++i) {
      ep[k][0] = pw[i][0] + pw[j][0];
      ep[k][1] = pw[i][1] + pw[j][1];
      ++k;
    }
  // S pass: slots = distinct axis-0 exponents of the ones channel
  memset(&t->s_col, 0, sizeof(ColArgs));
  memset(&t->t_col, 0, sizeof(ColArgs));
  memset(&t->s_row, 0, sizeof(RowArgs));
  memset(&t->t_row, 0, sizeof(RowArgs));
  int s_slot_of[9];
  for (int a = 0; a < 9; ++a) s_slot_of[a] = -1;
  int ns_slots = 0;
  for (int e = 0; e < t->ns; ++e) {
    int a0 = ep[e][0];
    if (s_slot_of[a0] < 0) {
      s_slot_of[a0] = ns_slots;
      t->s_col.slot_chan[ns_slots] = 0;
      t->s_col.slot_pow[ns_slots] = a0;
      ++ns_slots;
    }
  }
  t->s_nslots = ns_slots;
  // elements of distinct exponents (the first of each), the rest copied
  int uq[55];
  int nu = 0;
  t->ndup = 0;
  for (int e = 0; e < t->ns; ++e) {
    int first = -1;
    for (int f = 0; f < nu; ++f)
      if (ep[uq[f]][0] == ep[e][0] && ep[uq[f]][1] == ep[e][1]) first = uq[f];
    if (first < 0) {
      uq[nu++] = e;
    } else {
      t->dup_src[t->ndup] = first;
      t->dup_dst[t->ndup] = e;
      ++t->ndup;
    }
  }
  int nj = 0;
  for (int u = 0; u < nu; u += 2) {
    if (nj >= kMaxJobs) return FLPR_ERR_ARG;
    const int e = uq[u];
    RowJob jb;
    jb.slot_a = (short)s_slot_of[ep[e][0]];
    jb.pow_a = (short)ep[e][1];
    jb.out_a = (short)e;
    if (u + 1 < nu) {
      const int e2 = uq[u + 1];
      jb.slot_b = (short)s_slot_of[ep[e2][0]];
      jb.pow_b = (short)ep[e2][1];
      jb.out_b = (short)e2;
    } else {
      jb.slot_b = -1;
      jb.pow_b = 0;
      jb.out_b = 0;
    }
    t->s_row.jobs[nj++] = jb;
  }
  t->s_row.njobs = nj;
  // T pass: slots (value channel c, axis-0 exponent of term i)
  int a0_slot[9];
  for (int a = 0; a < 9; ++a) a0_slot[a] = -1;
  int na0 = 0;
  for (int i = 0; i < nt; ++i)
    if (a0_slot[pw[i][0]] < 0) a0_slot[pw[i][0]] = na0++;
  if (C * na0 > kMaxSlots) return FLPR_ERR_ARG;
  for (int c = 0; c < C; ++c)
    for (int a = 0; a < 9; ++a)
      if (a0_slot[a] >= 0) {
        const int sl = c * na0 + a0_slot[a];
        t->t_col.slot_chan[sl] = 1 + c;
        t->t_col.slot_pow[sl] = a;
      }
  t->t_nslots = C * na0;
  const int nprod = C * nt;
  nj = 0;
  for (int p = 0; p < nprod; p += 2) {
    if (nj >= kMaxJobs) return FLPR_ERR_ARG;
    const int c = p / nt, i = p - c * nt;
    RowJob jb;
    jb.slot_a = (short)(c * na0 + a0_slot[pw[i][0]]);
    jb.pow_a = (short)pw[i][1];
    jb.out_a = (short)p;
    if (p + 1 < nprod) {
      const int c2 = (p + 1) / nt, i2 = (p + 1) - c2 * nt;
      jb.slot_b = (short)(c2 * na0 + a0_slot[pw[i2][0]]);
      jb.pow_b = (short)pw[i2][1];
      jb.out_b = (short)(p + 1);
    } else {
      jb.slot_b = -1;
      jb.pow_b = 0;
      jb.out_b = 0;
    }
    t->t_row.jobs[nj++] = jb;
  }
  t->t_row.njobs = nj;
  return FLPR_OK;
}

static bool pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }


struct FusedGeom {
  int L0, L1, L1h, G0, G1, q0, q1;
  int64_t M;
  int Hc_s, Hc_t;
  size_t w_elems;
};

// vsize: bytes of one complex value of the passes (8 FP32, 16 FP64).
static int fused_geom(const int* G, const int* L, const int* qout, int H, const FusedTables& t,
                      size_t vsize, FusedGeom* fg) {
  fg->L0 = L[0];
  fg->L1 = L[1];
  fg->L1h = L[1] / 2 + 1;
  fg->G0 = G[0];
  fg->G1 = G[1];
  fg->q0 = qout[0];
  fg->q1 = qout[1];
  fg->M = (int64_t)G[0] * G[1];
  const size_t slab = (size_t)fg->G0 * fg->L1h;  // complex values per (slot, h)
  // chunks of a few bandwidths: enough row-pass CTAs to fill the GPU with a
  // bounded column-pass output (FLPR_TUNE_FUSED_CHUNK_MB)
  size_t budget = (size_t)tuning(FLPR_TUNE_FUSED_CHUNK_MB) << 20;
  const size_t budget_s = budget, budget_t = budget;
  int hs = (int)(budget_s / (vsize * slab * t.s_nslots));
  int ht = (int)(budget_t / (vsize * slab * t.t_nslots));
  fg->Hc_s = hs < 1 ? 1 : (hs > H ? H : hs);
  fg->Hc_t = ht < 1 ? 1 : (ht > H ? H : ht);
  // the same number of chunks, filled evenly (5 bandwidths: 3 + 2, not 4 + 1)
  fg->Hc_s = (H + (H + fg->Hc_s - 1) / fg->Hc_s - 1) / ((H + fg->Hc_s - 1) / fg->Hc_s);
  fg->Hc_t = (H + (H + fg->Hc_t - 1) / fg->Hc_t - 1) / ((H + fg->Hc_t - 1) / fg->Hc_t);
  size_t ws = slab * t.s_nslots * fg->Hc_s;
  size_t wt = slab * t.t_nslots * fg->Hc_t;
  fg->w_elems = ws > wt ? ws : wt;
  return FLPR_OK;
}

// Workspace carve-up, shared by the size query and the run.
template <typename T>
struct FusedBuffers {
  using V = typename Vec2<T>::V;
  V *Yt, *W, *tab0, *tab1, *Ff;
  double *z, *dpart;
  int* kcut;
};

template <typename T, typename A>
static void carve(A& ar, const FusedTables& tb, const FusedGeom& fg, int H, int npow, int C,
                  FusedBuffers<T>* b) {
  using V = typename Vec2<T>::V;
  b->Yt = ar.template take<V>((size_t)(1 + C) * fg.L1h * fg.L0);
  b->W = ar.template take<V>(fg.w_elems);
  b->tab0 = ar.template take<V>(twiddle_entries(fg.L0));
  b->tab1 = ar.template take<V>(twiddle_entries(fg.L1));
  b->Ff = ar.template take<V>((size_t)H * npow * (fg.L0 + fg.L1));
  b->z = ar.template take<double>((size_t)H * fg.M * tb.nt);
  b->dpart = ar.template take<double>((size_t)C * H * fg.G0);
  b->kcut = ar.template take<int>(2 * (size_t)H);
}

// Passes of one launch sequence: the S planes only (kSPass), the T pass on
// S planes given in FP64 with lambda already in `scalar` (kTPass), or both
// with lambda taken from the S planes (kBoth).
enum FusedMode { kBoth = 0, kSPass = 1, kTPass = 2 };

// S: the S planes (ns, H, M) in the pass precision (written by the S pass);
// S64: FP64 S planes given to the T pass (kTPass).
template <int E0, int E1, typename T>
static int run_fused(int mode, const FusedTables& tb, const FusedGeom& fg, int H, int npow,
                     int order, int C, int ny, const typename Vec2<T>::V* spec, const double2* F,
                     double scale, const double* Q, double reg, T* S, const double* S64,
                     double* my, double* dots, double* scalar, const double* scalar_floor_in,
                     const FusedBuffers<T>& b, cudaStream_t s) {
  using V = typename Vec2<T>::V;
  const int nt = tb.nt;
  twiddle_table_kernel<V><<<(twiddle_entries(fg.L0) + 255) / 256, 256, 0, s>>>(fg.L0, b.tab0);
  FLPR_LAUNCH_CHECK();
  twiddle_table_kernel<V><<<(twiddle_entries(fg.L1) + 255) / 256, 256, 0, s>>>(fg.L1, b.tab1);
  FLPR_LAUNCH_CHECK();
  {
    const int64_t n0 = (int64_t)H * npow * fg.L0, ntot = (int64_t)H * npow * (fg.L0 + fg.L1);
    int nb = (int)((ntot + 255) / 256);
    if (nb > 4 * sm_count()) nb = 4 * sm_count();
    factor_kernel<V><<<nb, 256, 0, s>>>(n0, ntot, scale, F, b.Ff);
    FLPR_LAUNCH_CHECK();
  }
  band_limit_kernel<<<dim3(H, 2), 256, 0, s>>>(H, npow, fg.L0, fg.L1, F,
                                                sizeof(T) == 4 ? kBandEps : kBandEps64, b.kcut);
  FLPR_LAUNCH_CHECK();
  const int* kcut1 = b.kcut + H;
  const V* F0f = b.Ff;
  const V* F1f = b.Ff + (size_t)H * npow * fg.L0;
  const int nspec = mode == kSPass ? 1 : 1 + C;
  transpose_spec_kernel<V><<<dim3((fg.L1h + 31) / 32, (fg.L0 + 31) / 32, nspec), dim3(32, 8), 0,
                             s>>>(nspec, fg.L0, fg.L1h, spec, b.Yt);
  FLPR_LAUNCH_CHECK();
  const int ncolblk = (fg.L1h + kColWarps - 1) / kColWarps;
  // S pass
  ColArgs ca = tb.s_col;
  ca.L0 = fg.L0;
  ca.L1h = fg.L1h;
  ca.G0 = fg.G0;
  ca.q0 = fg.q0;
  ca.npow = npow;
  ca.nslots = tb.s_nslots;
  RowArgs ra = tb.s_row;
  ra.L1 = fg.L1;
  ra.L1h = fg.L1h;
  ra.G0 = fg.G0;
  ra.G1 = fg.G1;
  ra.q1 = fg.q1;
  ra.npow = npow;
  if (mode != kTPass) {
    for (int h0 = 0; h0 < H; h0 += fg.Hc_s) {
      const int hc = H - h0 < fg.Hc_s ? H - h0 : fg.Hc_s;
      ca.hbase = h0;
      ra.hbase = h0;
      FLPR_TRY((launch_col<E0, T>(ca, ncolblk, tb.s_nslots, hc, b.Yt, F0f, b.tab0, kcut1, b.W,
                                           s)));
      FLPR_TRY((launch_row_s<E1, T>(ra, hc, H, hc, b.W, F1f, b.tab1, kcut1, S, s)));
    }
    for (int k = 0; k < tb.ndup; ++k)
      FLPR_CUDA(cudaMemcpyAsync(S + (size_t)tb.dup_dst[k] * H * fg.M,
                                S + (size_t)tb.dup_src[k] * H * fg.M,
                                sizeof(T) * (size_t)H * fg.M, cudaMemcpyDeviceToDevice, s));
    if (mode == kSPass) return FLPR_OK;
    FLPR_TRY(global_scalar(order, nt, H, fg.M, S, scalar,
                           sizeof(T) == 4 ? FLPR_PREC_F32 : FLPR_PREC_F64, s));
    FLPR_TRY(scalar_floor(scalar, scalar_floor_in, s));
  }
  {
    const int64_t HM = (int64_t)H * fg.M;
    int nb = (int)((HM + 255) / 256);
    if (nb > 16 * sm_count()) nb = 16 * sm_count();
#define FLPR_ZVEC(NTV)                                                                  \
  if (S64)                                                                              \
    zvec_kernel<NTV, double><<<nb, 256, 0, s>>>(order, H, fg.M, S64, scalar, reg, b.z); \
  else                                                                                  \
    zvec_kernel<NTV, T><<<nb, 256, 0, s>>>(order, H, fg.M, S, scalar, reg, b.z);
    switch (nt) {
      case 1: FLPR_ZVEC(1) break;
      case 3: FLPR_ZVEC(3) break;
      case 6: FLPR_ZVEC(6) break;
      default: set_error("fused2d: nt=%d", nt); return FLPR_ERR_ARG;
    }
#undef FLPR_ZVEC
    FLPR_LAUNCH_CHECK();
  }
  // T pass fused with the solve
  ca = tb.t_col;
  ca.L0 = fg.L0;
  ca.L1h = fg.L1h;
  ca.G0 = fg.G0;
  ca.q0 = fg.q0;
  ca.npow = npow;
  ca.nslots = tb.t_nslots;
  ra = tb.t_row;
  ra.L1 = fg.L1;
  ra.L1h = fg.L1h;
  ra.G0 = fg.G0;
  ra.G1 = fg.G1;
  ra.q1 = fg.q1;
  ra.npow = npow;
  for (int h0 = 0; h0 < H; h0 += fg.Hc_t) {
    const int hc = H - h0 < fg.Hc_t ? H - h0 : fg.Hc_t;
    ca.hbase = h0;
    ra.hbase = h0;
    FLPR_TRY((launch_col<E0, T>(ca, ncolblk, tb.t_nslots, hc, b.Yt, F0f, b.tab0, kcut1, b.W,
                                         s)));
    FLPR_TRY(launch_row_t<E1>(nt, ra, hc, H, hc, b.W, F1f, b.tab1, kcut1, C, ny, b.z, Q, my,
                              b.dpart, s));
  }
  dots_reduce_kernel<<<C * H, 256, 0, s>>>(C * H, fg.G0, b.dpart, dots);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int E0, typename T>
static int dispatch_e1(int mode, int E1, const FusedTables& tb, const FusedGeom& fg, int H,
                       int npow, int order, int C, int ny, const typename Vec2<T>::V* spec,
                       const double2* F, double scale, const double* Q, double reg, T* S,
                       const double* S64, double* my, double* dots, double* scalar,
                       const double* floor_in, const FusedBuffers<T>& b, cudaStream_t s) {
#define FLPR_E1(V)                                                                           \
  case V:                                                                                    \
    return run_fused<E0, V, T>(mode, tb, fg, H, npow, order, C, ny, spec, F, scale, Q, reg, \
                               S, S64, my, dots, scalar, floor_in, b, s);
  switch (E1) {
    FLPR_E1(2)
    FLPR_E1(4)
    FLPR_E1(8)
    FLPR_E1(16)
    FLPR_E1(32)
    default:
      set_error("fused2d: unsupported L1");
      return FLPR_ERR_ARG;
  }
#undef FLPR_E1
}

}  // namespace

int fused2d_check(int prec, const int* G, const int* L, const int* qout, int H, int order, int C,
                  FusedTables* tb, FusedGeom* fg) {
  FLPR_CHECK_ARG(prec == FLPR_PREC_F32 || prec == FLPR_PREC_F64, "fused2d: precision %d", prec);
  const bool f64 = prec == FLPR_PREC_F64;
  FLPR_CHECK_ARG(pow2_in(L[0], 64, 1024) && pow2_in(L[1], 64, 1024),
                 "fused2d: L=(%d,%d) must be powers of two in [64, 1024]", L[0], L[1]);
  FLPR_CHECK_ARG(G[0] >= 2 && G[1] >= 2 && G[0] <= L[0] && G[1] <= L[1], "fused2d: G");
  FLPR_CHECK_ARG(qout[0] >= 0 && qout[0] + G[0] <= L[0] && qout[1] >= 0 && qout[1] + G[1] <= L[1],
                 "fused2d: crop window");
  // a warp's cropped output (2 G reals) must fit its transpose buffer
  const int b0 = f64 ? warp_buf_stride64(L[0] / 32) : warp_buf_stride(L[0] / 32);
  const int b1 = f64 ? warp_buf_stride64(L[1] / 32) : warp_buf_stride(L[1] / 32);
  FLPR_CHECK_ARG(2 * G[0] <= b0 && 2 * G[1] <= b1,
                 "fused2d: grid (%d,%d) too large for padding (%d,%d)", G[0], G[1], L[0], L[1]);
  FLPR_CHECK_ARG(order >= 0 && order <= 2 && C >= 1 && C <= 32 && H >= 1, "fused2d: order/C/H");
  FLPR_CHECK_ARG(build_tables(order, C, tb) == FLPR_OK, "fused2d: too many slots or jobs");
  const int nwarps = t_warps(tb->t_row.njobs);
  const size_t tsm = f64 ? t_smem_bytes<double>(L[1] / 32, nwarps, tb->t_row.njobs, G[1])
                         : t_smem_bytes<float>(L[1] / 32, nwarps, tb->t_row.njobs, G[1]);
  FLPR_CHECK_ARG(tsm <= kMaxSmem, "fused2d: T row tile does not fit shared memory");
  const size_t psm = f64 ? warp_pass_smem<double>(L[0] / 32, kColWarps)
                         : warp_pass_smem<float>(L[0] / 32, kColWarps);
  FLPR_CHECK_ARG(psm <= kMaxSmem, "fused2d: column tile does not fit shared memory");
  // a channel's products span at most two consecutive T rounds
  FLPR_CHECK_ARG(tb->t_row.njobs <= kTWarps || tb->nt <= 2 * kTWarps + 1,
                 "fused2d: %d terms per channel span more than two T rounds", tb->nt);
  fused_geom(G, L, qout, H, *tb, f64 ? sizeof(double2) : sizeof(float2), fg);
  return FLPR_OK;
}

}  // namespace flpr

using namespace flpr;

namespace {

template <typename T>
size_t fused_ws_bytes(const FusedTables& tb, const FusedGeom& fg, int H, int npow, int C) {
  ArenaSize ar;
  FusedBuffers<T> b;
  carve<T>(ar, tb, fg, H, npow, C, &b);
  return ar.used;
}

template <typename T>
int fused_run_t(int mode, const FusedTables& tb, const FusedGeom& fg, int H, int npow, int order,
                int C, int ny, const void* d_spec, const void* d_F, double scale,
                const double* d_Q, double reg, void* d_S, const double* d_S64, double* d_my,
                double* d_dots, double* d_scalar, const double* d_scalar_floor, void* d_ws,
                size_t ws_bytes, cudaStream_t s) {
  using V = typename Vec2<T>::V;
  const size_t need = fused_ws_bytes<T>(tb, fg, H, npow, C);
  if (ws_bytes < need) {
    set_error("fused2d: workspace too small (%zu < %zu)", ws_bytes, need);
    return FLPR_ERR_WORKSPACE;
  }
  Arena ar(d_ws, ws_bytes);
  FusedBuffers<T> b;
  carve<T>(ar, tb, fg, H, npow, C, &b);
  const V* spec = static_cast<const V*>(d_spec);
  const double2* F = static_cast<const double2*>(d_F);
  T* S = static_cast<T*>(d_S);
  switch (fg.L0 / 32) {
#define FLPR_E0(EV)                                                                           \
  case EV:                                                                                    \
    return dispatch_e1<EV, T>(mode, fg.L1 / 32, tb, fg, H, npow, order, C, ny, spec, F, scale, \
                              d_Q, reg, S, d_S64, d_my, d_dots, d_scalar, d_scalar_floor, b, s);
    FLPR_E0(2)
    FLPR_E0(4)
    FLPR_E0(8)
    FLPR_E0(16)
    FLPR_E0(32)
#undef FLPR_E0
    default:
      set_error("fused2d: unsupported L0");
      return FLPR_ERR_ARG;
  }
}

}  // namespace

extern "C" {

int flpr_lpr2d_fused_ex_supported(int prec, const int* h_G, const int* h_L, const int* h_qout,
                                  int H, int order, int C) {
  FusedTables tb;
  FusedGeom fg;
  return fused2d_check(prec, h_G, h_L, h_qout, H, order, C, &tb, &fg) == FLPR_OK ? 1 : 0;
}

size_t flpr_lpr2d_fused_ex_ws(int prec, const int* h_G, const int* h_L, const int* h_qout, int H,
                              int order, int C) {
  FusedTables tb;
  FusedGeom fg;
  if (fused2d_check(prec, h_G, h_L, h_qout, H, order, C, &tb, &fg) != FLPR_OK) return 0;
  return prec == FLPR_PREC_F64 ? fused_ws_bytes<double>(tb, fg, H, 2 * order + 1, C)
                               : fused_ws_bytes<float>(tb, fg, H, 2 * order + 1, C);
}

int flpr_lpr2d_fused_ex(int prec, int mode, const int* h_G, const int* h_L, const int* h_qout,
                        int H, int npow, int order, int C, int ny, const void* d_spec,
                        const void* d_F, double scale, const double* d_Q, double reg, void* d_S,
                        const double* d_S64, double* d_my, double* d_dots, double* d_scalar,
                        const double* d_scalar_floor, void* d_ws, size_t ws_bytes, void* stream) {
  FusedTables tb;
  FusedGeom fg;
  FLPR_TRY(fused2d_check(prec, h_G, h_L, h_qout, H, order, C, &tb, &fg));
  FLPR_CHECK_ARG(mode == kBoth || mode == kSPass || mode == kTPass, "fused2d: mode %d", mode);
  FLPR_CHECK_ARG(ny >= 0 && ny <= C, "fused2d: ny=%d", ny);
  FLPR_CHECK_ARG(npow >= 2 * order + 1, "fused2d: npow=%d < 2*order+1", npow);
  FLPR_CHECK_ARG(d_spec != nullptr && d_F != nullptr, "fused2d: spectra or factors missing");
  if (mode != kTPass) FLPR_CHECK_ARG(d_S != nullptr, "fused2d: S planes missing");
  if (mode == kTPass)
    FLPR_CHECK_ARG(d_S64 != nullptr && d_scalar != nullptr, "fused2d: S planes or scalar missing");
  if (mode != kSPass)
    FLPR_CHECK_ARG(d_Q != nullptr && d_dots != nullptr && d_scalar != nullptr &&
                       (ny == 0 || d_my != nullptr),
                   "fused2d: T-pass outputs missing");
  cudaStream_t s = as_stream(stream);
  if (prec == FLPR_PREC_F64)
    return fused_run_t<double>(mode, tb, fg, H, npow, order, C, ny, d_spec, d_F, scale, d_Q, reg,
                               d_S, mode == kTPass ? d_S64 : nullptr, d_my, d_dots, d_scalar,
                               d_scalar_floor, d_ws, ws_bytes, s);
  return fused_run_t<float>(mode, tb, fg, H, npow, order, C, ny, d_spec, d_F, scale, d_Q, reg,
                            d_S, mode == kTPass ? d_S64 : nullptr, d_my, d_dots, d_scalar,
                            d_scalar_floor, d_ws, ws_bytes, s);
}

int flpr_lpr2d_fused_supported(const int* h_G, const int* h_L, const int* h_qout, int H, int order,
                               int C) {
  return flpr_lpr2d_fused_ex_supported(FLPR_PREC_F32, h_G, h_L, h_qout, H, order, C);
}

size_t flpr_lpr2d_fused_ws(const int* h_G, const int* h_L, const int* h_qout, int H, int order,
                           int C) {
  return flpr_lpr2d_fused_ex_ws(FLPR_PREC_F32, h_G, h_L, h_qout, H, order, C);
}

int flpr_lpr2d_fused_floor(const int* h_G, const int* h_L, const int* h_qout, int H, int npow,
                           int order, int C, int ny, const void* d_spec, const void* d_F,
                           double scale, const double* d_Q, double reg, float* d_S, double* d_my,
                           double* d_dots, double* d_scalar, const double* d_scalar_floor,
                           void* d_ws, size_t ws_bytes, void* stream) {
  return flpr_lpr2d_fused_ex(FLPR_PREC_F32, kBoth, h_G, h_L, h_qout, H, npow, order, C, ny,
                             d_spec, d_F, scale, d_Q, reg, d_S, nullptr, d_my, d_dots, d_scalar,
                             d_scalar_floor, d_ws, ws_bytes, stream);
}

int flpr_lpr2d_fused(const int* h_G, const int* h_L, const int* h_qout, int H, int npow, int order,
                     int C, int ny, const void* d_spec, const void* d_F, double scale,
                     const double* d_Q, double reg, float* d_S, double* d_my, double* d_dots,
                     double* d_scalar, void* d_ws, size_t ws_bytes, void* stream) {
  return flpr_lpr2d_fused_floor(h_G, h_L, h_qout, H, npow, order, C, ny, d_spec, d_F, scale, d_Q,
                                reg, d_S, d_my, d_dots, d_scalar, nullptr, d_ws, ws_bytes, stream);
}

int flpr_lpr2d_fused_t(const int* h_G, const int* h_L, const int* h_qout, int H, int npow,
                       int order, int C, int ny, const void* d_spec, const void* d_F, double scale,
                       const double* d_Q, double reg, const double* d_S64, const double* d_scalar,
                       double* d_my, double* d_dots, void* d_ws, size_t ws_bytes, void* stream) {
  return flpr_lpr2d_fused_ex(FLPR_PREC_F32, kTPass, h_G, h_L, h_qout, H, npow, order, C, ny,
                             d_spec, d_F, scale, d_Q, reg, nullptr, d_S64, d_my, d_dots,
                             const_cast<double*>(d_scalar), nullptr, d_ws, ws_bytes, stream);
}

}  // extern "C"
