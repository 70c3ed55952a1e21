// Fused 2-D FP32 convolution + solve for the LPR GCV sweep.
//
// The Gaussian kernel spectrum is separable, K(w0, w1) = A0(w0) A1(w1), so
// the inverse transform of every product Y_c K splits into
//   column pass: W_{c,a0,h}(x0, w1) = IFFT_0(Y_c(., w1) A0_{h,a0})(x0), x0 cropped,
//   row pass:    r(x0, x1) = C2R_1(W(x0, .) A1_{h,a1})(x1), x1 cropped,
// and W is shared by every moment element with the same axis-0 exponent.
// Each 1-D transform is one warp: a radix-2 DIF over the E = N/32 elements a
// lane holds (n = 32 s + lane), a twiddle step, and a 32-point DIF across the
// lanes with shuffles.  Two real row products share one complex transform
// (both spectra are Hermitian).  The row pass of the T elements is fused
// with the per-point FP64 solve and the dual-form reductions, so neither the
// T planes nor the probe fits touch HBM.
#include "common.cuh"
#include "linalg.cuh"
#include "plans.cuh"

namespace flpr {

int global_scalar(int order, int nt, int H, int64_t M, const void* d_S, double* d_scalar, int prec,
                  cudaStream_t s);

size_t fused_t_smem(int E, int G1, int nt, int C);

namespace {

constexpr int kFusedThreads = 256;
constexpr int kColBlock = 8;     // columns per column-pass CTA (one per warp)
constexpr int kMaxSlots = 64;
constexpr int kMaxJobs = 64;

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__host__ __device__ constexpr int brev(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r = (r << 1) | ((x >> i) & 1);
  return r;
}
__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

// Inverse (unnormalised) FFT of length N = 32 E held by one warp: on entry
// lane l, slot s holds x[32 s + l]; on exit it holds X[brev_E(s) + E brev_5(l)].
// tw[k] = exp(2 pi i k / N); tw2[k1 * 32 + l] = exp(2 pi i l k1 / N).
template <int E>
__device__ __forceinline__ void warp_ifft(float2 (&v)[E], const float2* __restrict__ tw,
                                          const float2* __restrict__ tw2, int lane) {
  constexpr int N = 32 * E;
  constexpr int EB = ilog2(E);
#pragma unroll
  for (int span = E / 2; span >= 1; span >>= 1) {
#pragma unroll
    for (int s = 0; s < E; ++s) {
      if ((s & span) == 0) {
        const int i = s & (span - 1);
        const float2 a = v[s], b = v[s + span];
        v[s] = cadd(a, b);
        v[s + span] = i == 0 ? csub(a, b) : cmul(csub(a, b), tw[i * (N / (2 * span))]);
      }
    }
  }
#pragma unroll
  for (int s = 0; s < E; ++s) v[s] = cmul(v[s], tw2[brev(s, EB) * 32 + lane]);
#pragma unroll
  for (int span = 16; span >= 1; span >>= 1) {
    const bool upper = (lane & span) != 0;
    const float2 w = tw[(lane & (span - 1)) * (N / (2 * span))];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      float2 p;
      p.x = __shfl_xor_sync(0xffffffffu, v[s].x, span);
      p.y = __shfl_xor_sync(0xffffffffu, v[s].y, span);
      v[s] = upper ? cmul(csub(p, v[s]), w) : cadd(v[s], p);
    }
  }
}

// tables for length N (tw: N entries, tw2: 32*N/32 entries) in global memory
__global__ void twiddle_table_kernel(int N, float2* tw, float2* tw2) {
  const int E = N / 32;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi(2.0 * (double)k / (double)N, &sn, &cs);
    tw[k] = make_float2((float)cs, (float)sn);
    const int k1 = k / 32, l = k % 32;
    if (k1 < E) {
      sincospi(2.0 * (double)((l * k1) % N) / (double)N, &sn, &cs);
      tw2[k] = make_float2((float)cs, (float)sn);
    }
  }
}

template <int E>
__device__ __forceinline__ void load_twiddles(float2* s_tw, float2* s_tw2, const float2* tw,
                                              const float2* tw2) {
  constexpr int N = 32 * E;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    s_tw[i] = tw[i];
    s_tw2[i] = tw2[i];
  }
}

// (C, L0, L1h) -> (C, L1h, L0)
__global__ void transpose_spec_kernel(int C, int L0, int L1h, const float2* __restrict__ in,
                                      float2* __restrict__ out) {
  __shared__ float2 tile[32][33];
  const int c = blockIdx.z;
  const int w0 = blockIdx.y * 32, w1 = blockIdx.x * 32;
  const float2* src = in + (size_t)c * L0 * L1h;
  float2* dst = out + (size_t)c * L0 * L1h;
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
  double scale;
  int slot_chan[kMaxSlots];
  int slot_pow[kMaxSlots];
};

// grid (ceil(L1h/8), nslots, Hc); warp w handles column blockIdx.x*8+w.
// W layout: [slot][hz][r][w1], r = x0 - q0 in [0, G0).
template <int E>
__global__ void __launch_bounds__(kFusedThreads, 3)
colpass_kernel(ColArgs ca, const float2* __restrict__ Yt, const double2* __restrict__ F0,
               const float2* __restrict__ tw, const float2* __restrict__ tw2,
               float2* __restrict__ W) {
  constexpr int N = 32 * E;
  constexpr int EB = ilog2(E);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* s_tw = reinterpret_cast<float2*>(smem_raw);
  float2* s_tw2 = s_tw + N;
  float2* stage = s_tw2 + N;  // G0 x 8
  load_twiddles<E>(s_tw, s_tw2, tw, tw2);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = blockIdx.y, hz = blockIdx.z, h = ca.hbase + hz;
  const int c = ca.slot_chan[slot], a0 = ca.slot_pow[slot];
  const int w1 = blockIdx.x * kColBlock + warp;
  if (w1 < ca.L1h) {
    const float2* col = Yt + ((size_t)c * ca.L1h + w1) * N;
    const double2* f = F0 + ((size_t)h * ca.npow + a0) * N;
    float2 v[E];
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int k = 32 * s + lane;
      const double2 fv = f[k];
      const float2 y = col[k];
      v[s] = cmul(y, make_float2((float)(fv.x * ca.scale), (float)(fv.y * ca.scale)));
    }
    warp_ifft<E>(v, s_tw, s_tw2, lane);
#pragma unroll
    for (int s = 0; s < E; ++s) {
      const int r = brev(s, EB) + E * brev(lane, 5) - ca.q0;
      if (r >= 0 && r < ca.G0) stage[r * kColBlock + warp] = v[s];
    }
  }
  __syncthreads();
  float2* out = W + ((size_t)slot * gridDim.z + hz) * ca.G0 * ca.L1h;
  for (int i = threadIdx.x; i < ca.G0 * kColBlock; i += blockDim.x) {
    const int r = i / kColBlock, wl = i - r * kColBlock;
    const int col = blockIdx.x * kColBlock + wl;
    if (col < ca.L1h) out[(size_t)r * ca.L1h + col] = stage[i];
  }
}

// Solve vectors z = (S + lam I)^-1 e1 per (bandwidth, grid point); order 0
// stores 1/max(s, max(s) reg).  S: (ns, H, M) float; z: (H, M, NT) double.
template <int NT>
__global__ void zvec_kernel(int order, int H, int64_t M, const float* __restrict__ S,
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

// Hermitian-extended spectrum value k of product W_row * A1 (k in [0, L1)).
__device__ __forceinline__ float2 herm_product(const float2* __restrict__ wrow,
                                               const double2* __restrict__ f, int k, int N) {
  const bool mirror = k > N / 2;
  const int kk = mirror ? N - k : k;
  const float2 w = wrow[kk];
  const double2 a = f[kk];
  float2 p = cmul(w, make_float2((float)a.x, (float)a.y));
  if (kk == 0 || 2 * kk == N) p.y = 0.0f;
  if (mirror) p.y = -p.y;
  return p;
}

// One warp computes the products of one job for row r and leaves the cropped
// real results (x1 - q1 in [0, G1)) in out_a / out_b (shared memory rows).
template <int E>
__device__ __forceinline__ void row_job(const RowArgs& ra, const RowJob& jb, int r, int hz, int h,
                                        int nslots_w, const float2* __restrict__ W,
                                        const double2* __restrict__ F1, const float2* s_tw,
                                        const float2* s_tw2, int lane, float* out_a,
                                        float* out_b) {
  constexpr int N = 32 * E;
  constexpr int EB = ilog2(E);
  const size_t rowstride = (size_t)ra.L1h;
  const float2* wa = W + (((size_t)jb.slot_a * nslots_w + hz) * ra.G0 + r) * rowstride;
  const double2* fa = F1 + ((size_t)h * ra.npow + jb.pow_a) * N;
  const bool pair = jb.slot_b >= 0;
  const float2* wb = pair ? W + (((size_t)jb.slot_b * nslots_w + hz) * ra.G0 + r) * rowstride : wa;
  const double2* fb = pair ? F1 + ((size_t)h * ra.npow + jb.pow_b) * N : fa;
  float2 v[E];
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int k = 32 * s + lane;
    const float2 pa = herm_product(wa, fa, k, N);
    float2 z = pa;
    if (pair) {
      const float2 pb = herm_product(wb, fb, k, N);
      z = make_float2(pa.x - pb.y, pa.y + pb.x);
    }
    v[s] = z;
  }
  warp_ifft<E>(v, s_tw, s_tw2, lane);
#pragma unroll
  for (int s = 0; s < E; ++s) {
    const int x = brev(s, EB) + E * brev(lane, 5) - ra.q1;
    if (x >= 0 && x < ra.G1) {
      out_a[x] = v[s].x;
      if (pair) out_b[x] = v[s].y;
    }
  }
}

// S pass: grid (G0, Hc).  S planes (ns, H, G0*G1) float.
template <int E>
__global__ void __launch_bounds__(kFusedThreads, 2)
rowpass_s_kernel(RowArgs ra, int H, int nslots_w, const float2* __restrict__ W,
                 const double2* __restrict__ F1, const float2* __restrict__ tw,
                 const float2* __restrict__ tw2, float* __restrict__ S) {
  constexpr int N = 32 * E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* s_tw = reinterpret_cast<float2*>(smem_raw);
  float2* s_tw2 = s_tw + N;
  float* rows = reinterpret_cast<float*>(s_tw2 + N);  // (nwarps, 2, G1)
  load_twiddles<E>(s_tw, s_tw2, tw, tw2);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int r = blockIdx.x, hz = blockIdx.y, h = ra.hbase + hz;
  const int64_t M = (int64_t)ra.G0 * ra.G1;
  float* ra_row = rows + (size_t)warp * 2 * ra.G1;
  float* rb_row = ra_row + ra.G1;
  for (int j = warp; j < ra.njobs; j += nwarps) {
    const RowJob jb = ra.jobs[j];
    row_job<E>(ra, jb, r, hz, h, nslots_w, W, F1, s_tw, s_tw2, lane, ra_row, rb_row);
    __syncwarp();
    float* da = S + ((size_t)jb.out_a * H + h) * M + (size_t)r * ra.G1;
    for (int x = lane; x < ra.G1; x += 32) da[x] = ra_row[x];
    if (jb.slot_b >= 0) {
      float* db = S + ((size_t)jb.out_b * H + h) * M + (size_t)r * ra.G1;
      for (int x = lane; x < ra.G1; x += 32) db[x] = rb_row[x];
    }
    __syncwarp();
  }
}

// T pass fused with the solve and the dual-form reductions: grid (G0, Hc).
// Products (c, i) go to Tsm[c * nt + i][x1]; the solve vector z = (S+lam I)^-1 e1
// (order >= 1) or 1/max(s, thr) (order 0) per x1; m_c = sum_i z_i T_ci.
template <int E>
__global__ void __launch_bounds__(kFusedThreads, 2)
rowpass_t_solve_kernel(RowArgs ra, int H, int nslots_w, const float2* __restrict__ W,
                       const double2* __restrict__ F1, const float2* __restrict__ tw,
                       const float2* __restrict__ tw2, int nt, int C, int ny,
                       const double* __restrict__ zg, const double* __restrict__ Q,
                       double* __restrict__ my, double* __restrict__ dots) {
  constexpr int N = 32 * E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* s_tw = reinterpret_cast<float2*>(smem_raw);
  float2* s_tw2 = s_tw + N;
  double* zsm = reinterpret_cast<double*>(s_tw2 + N);          // G1 x nt
  float* Tsm = reinterpret_cast<float*>(zsm + (size_t)ra.G1 * nt);  // (C*nt) x G1
  __shared__ double red[kFusedThreads / 32];
  load_twiddles<E>(s_tw, s_tw2, tw, tw2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int r = blockIdx.x, hz = blockIdx.y, h = ra.hbase + hz;
  const int64_t M = (int64_t)ra.G0 * ra.G1;
  // phase 1: the row's solve vectors
  {
    const double* src = zg + ((int64_t)h * M + (int64_t)r * ra.G1) * nt;
    for (int i = threadIdx.x; i < ra.G1 * nt; i += blockDim.x) zsm[i] = src[i];
  }
  __syncthreads();
  // phase 2: T products
  for (int j = warp; j < ra.njobs; j += nwarps) {
    const RowJob jb = ra.jobs[j];
    float* oa = Tsm + (size_t)jb.out_a * ra.G1;
    float* ob = jb.slot_b >= 0 ? Tsm + (size_t)jb.out_b * ra.G1 : oa;
    row_job<E>(ra, jb, r, hz, h, nslots_w, W, F1, s_tw, s_tw2, lane, oa, ob);
  }
  __syncthreads();
  // phase 3: m, fitted grids, dots
  for (int c = 0; c < C; ++c) {
    double acc = 0.0;
    for (int x = threadIdx.x; x < ra.G1; x += blockDim.x) {
      const double* z = zsm + (size_t)x * nt;
      double m = 0.0;
      for (int i = 0; i < nt; ++i) m += z[i] * (double)Tsm[(size_t)(c * nt + i) * ra.G1 + x];
      const int64_t g = (int64_t)r * ra.G1 + x;
      if (c < ny) my[((int64_t)h * M + g) * ny + c] = m;
      acc += m * Q[g * C + c];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < nwarps; ++w) s += red[w];
      atomicAdd(&dots[(int64_t)c * H + h], s);
    }
    __syncthreads();
  }
}

}  // namespace

size_t fused_t_smem(int E, int G1, int nt, int C) {
  return sizeof(float2) * 2 * 32 * (size_t)E + sizeof(double) * (size_t)G1 * nt +
         sizeof(float) * (size_t)C * nt * G1;
}

namespace {

struct Plan2D {
  int L0, L1, L1h, G0, G1, q0, q1, E0, E1;
  int64_t M;
};

template <typename K>
static int set_smem(K kernel, size_t bytes) {
  FLPR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  // let several CTAs share an SM: take the whole unified L1/shared array as shared memory
  FLPR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
  return FLPR_OK;
}

template <int E>
static int launch_col(const ColArgs& ca, int ncolblk, int nslots, int Hc, const float2* Yt,
                      const double2* F0, const float2* tw, const float2* tw2, float2* W,
                      cudaStream_t s) {
  constexpr int N = 32 * E;
  size_t smem = sizeof(float2) * (2 * N + (size_t)ca.G0 * kColBlock);
  FLPR_TRY(set_smem(colpass_kernel<E>, smem));
  colpass_kernel<E><<<dim3(ncolblk, nslots, Hc), kFusedThreads, smem, s>>>(ca, Yt, F0, tw, tw2, W);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int E>
static int launch_row_s(const RowArgs& ra, int G0, int Hc, int H, int nslots_w, const float2* W,
                        const double2* F1, const float2* tw, const float2* tw2, float* S,
                        cudaStream_t s) {
  constexpr int N = 32 * E;
  size_t smem = sizeof(float2) * 2 * N + sizeof(float) * (kFusedThreads / 32) * 2 * ra.G1;
  FLPR_TRY(set_smem(rowpass_s_kernel<E>, smem));
  rowpass_s_kernel<E><<<dim3(G0, Hc), kFusedThreads, smem, s>>>(ra, H, nslots_w, W, F1, tw, tw2, S);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

template <int E>
static int launch_row_t(const RowArgs& ra, int G0, int Hc, int H, int nslots_w, const float2* W,
                        const double2* F1, const float2* tw, const float2* tw2, int nt, int C,
                        int ny, const double* z, const double* Q, double* my, double* dots,
                        cudaStream_t s) {
  size_t smem = fused_t_smem(E, ra.G1, nt, C);
  FLPR_TRY(set_smem(rowpass_t_solve_kernel<E>, smem));
  rowpass_t_solve_kernel<E><<<dim3(G0, Hc), kFusedThreads, smem, s>>>(
      ra, H, nslots_w, W, F1, tw, tw2, nt, C, ny, z, Q, my, dots);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

// Slot/job tables of one configuration.
struct FusedTables {
  int nt, ns;
  int s_nslots, t_nslots;
  ColArgs s_col, t_col;
  RowArgs s_row, t_row;
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
  int nj = 0;
  for (int e = 0; e < t->ns; e += 2) {
    if (nj >= kMaxJobs) return FLPR_ERR_ARG;
    RowJob jb;
    jb.slot_a = (short)s_slot_of[ep[e][0]];
    jb.pow_a = (short)ep[e][1];
    jb.out_a = (short)e;
    if (e + 1 < t->ns) {
      jb.slot_b = (short)s_slot_of[ep[e + 1][0]];
      jb.pow_b = (short)ep[e + 1][1];
      jb.out_b = (short)(e + 1);
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

static int fused_geom(const int* G, const int* L, const int* qout, int H, const FusedTables& t,
                      FusedGeom* fg) {
  fg->L0 = L[0];
  fg->L1 = L[1];
  fg->L1h = L[1] / 2 + 1;
  fg->G0 = G[0];
  fg->G1 = G[1];
  fg->q0 = qout[0];
  fg->q1 = qout[1];
  fg->M = (int64_t)G[0] * G[1];
  const size_t slab = (size_t)fg->G0 * fg->L1h;  // float2 per (slot, h)
  // T chunks of a few bandwidths: enough row-pass CTAs to fill the GPU while
  // the column-pass output stays near the L2 size
  const size_t budget_s = (size_t)256 << 20, budget_t = (size_t)192 << 20;
  int hs = (int)(budget_s / (sizeof(float2) * slab * t.s_nslots));
  int ht = (int)(budget_t / (sizeof(float2) * slab * t.t_nslots));
  fg->Hc_s = hs < 1 ? 1 : (hs > H ? H : hs);
  fg->Hc_t = ht < 1 ? 1 : (ht > H ? H : ht);
  size_t ws = slab * t.s_nslots * fg->Hc_s;
  size_t wt = slab * t.t_nslots * fg->Hc_t;
  fg->w_elems = ws > wt ? ws : wt;
  return FLPR_OK;
}

template <int E0, int E1>
static int run_fused(const FusedTables& tb, const FusedGeom& fg, int H, int npow, int order, int C,
                     int ny, const float2* spec, const double2* F, double scale, const double* Q,
                     double reg, float* S, double* my, double* dots, double* scalar, float2* Yt,
                     float2* W, float2* tw0, float2* tw20, float2* tw1, float2* tw21,
                     double* zbuf, cudaStream_t s) {
  const int nt = tb.nt;
  const double2* F0 = F;
  const double2* F1 = F + (size_t)H * npow * fg.L0;
  twiddle_table_kernel<<<(fg.L0 + 255) / 256, 256, 0, s>>>(fg.L0, tw0, tw20);
  FLPR_LAUNCH_CHECK();
  twiddle_table_kernel<<<(fg.L1 + 255) / 256, 256, 0, s>>>(fg.L1, tw1, tw21);
  FLPR_LAUNCH_CHECK();
  transpose_spec_kernel<<<dim3((fg.L1h + 31) / 32, (fg.L0 + 31) / 32, 1 + C), dim3(32, 8), 0, s>>>(
      1 + C, fg.L0, fg.L1h, spec, Yt);
  FLPR_LAUNCH_CHECK();
  const int ncolblk = (fg.L1h + kColBlock - 1) / kColBlock;
  // S pass
  ColArgs ca = tb.s_col;
  ca.L0 = fg.L0;
  ca.L1h = fg.L1h;
  ca.G0 = fg.G0;
  ca.q0 = fg.q0;
  ca.npow = npow;
  ca.nslots = tb.s_nslots;
  ca.scale = scale;
  RowArgs ra = tb.s_row;
  ra.L1 = fg.L1;
  ra.L1h = fg.L1h;
  ra.G0 = fg.G0;
  ra.G1 = fg.G1;
  ra.q1 = fg.q1;
  ra.npow = npow;
  for (int h0 = 0; h0 < H; h0 += fg.Hc_s) {
    const int hc = H - h0 < fg.Hc_s ? H - h0 : fg.Hc_s;
    ca.hbase = h0;
    ra.hbase = h0;
    FLPR_TRY(launch_col<E0>(ca, ncolblk, tb.s_nslots, hc, Yt, F0, tw0, tw20, W, s));
    FLPR_TRY(launch_row_s<E1>(ra, fg.G0, hc, H, hc, W, F1, tw1, tw21, S, s));
  }
  FLPR_TRY(global_scalar(order, nt, H, fg.M, S, scalar, FLPR_PREC_F32, s));
  FLPR_CUDA(cudaMemsetAsync(dots, 0, sizeof(double) * (size_t)C * H, s));
  {
    const int64_t HM = (int64_t)H * fg.M;
    int nb = (int)((HM + 255) / 256);
    if (nb > 16 * sm_count()) nb = 16 * sm_count();
    switch (nt) {
      case 1: zvec_kernel<1><<<nb, 256, 0, s>>>(order, H, fg.M, S, scalar, reg, zbuf); break;
      case 3: zvec_kernel<3><<<nb, 256, 0, s>>>(order, H, fg.M, S, scalar, reg, zbuf); break;
      case 6: zvec_kernel<6><<<nb, 256, 0, s>>>(order, H, fg.M, S, scalar, reg, zbuf); break;
      default: set_error("fused2d: nt=%d", nt); return FLPR_ERR_ARG;
    }
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
  ca.scale = scale;
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
    FLPR_TRY(launch_col<E0>(ca, ncolblk, tb.t_nslots, hc, Yt, F0, tw0, tw20, W, s));
    FLPR_TRY(launch_row_t<E1>(ra, fg.G0, hc, H, hc, W, F1, tw1, tw21, nt, C, ny, zbuf, Q, my,
                              dots, s));
  }
  return FLPR_OK;
}

template <int E0>
static int dispatch_e1(int E1, const FusedTables& tb, const FusedGeom& fg, int H, int npow,
                       int order, int C, int ny, const float2* spec, const double2* F,
                       double scale, const double* Q, double reg, float* S, double* my,
                       double* dots, double* scalar, float2* Yt, float2* W, float2* tw0,
                       float2* tw20, float2* tw1, float2* tw21, double* zbuf, cudaStream_t s) {
#define FLPR_E1(V)                                                                            \
  case V:                                                                                     \
    return run_fused<E0, V>(tb, fg, H, npow, order, C, ny, spec, F, scale, Q, reg, S, my,     \
                            dots, scalar, Yt, W, tw0, tw20, tw1, tw21, zbuf, s);
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

int fused2d_check(const int* G, const int* L, const int* qout, int H, int order, int C,
                  FusedTables* tb, FusedGeom* fg) {
  FLPR_CHECK_ARG(pow2_in(L[0], 64, 1024) && pow2_in(L[1], 64, 1024),
                 "fused2d: L=(%d,%d) must be powers of two in [64, 1024]", L[0], L[1]);
  FLPR_CHECK_ARG(G[0] >= 2 && G[1] >= 2 && G[0] <= L[0] && G[1] <= L[1], "fused2d: G");
  FLPR_CHECK_ARG(qout[0] >= 0 && qout[0] + G[0] <= L[0] && qout[1] >= 0 && qout[1] + G[1] <= L[1],
                 "fused2d: crop window");
  FLPR_CHECK_ARG(order >= 0 && order <= 2 && C >= 1 && C <= 32 && H >= 1, "fused2d: order/C/H");
  FLPR_CHECK_ARG(build_tables(order, C, tb) == FLPR_OK, "fused2d: too many slots or jobs");
  FLPR_CHECK_ARG(fused_t_smem(L[1] / 32, G[1], tb->nt, C) <= 200 * 1024,
                 "fused2d: T tile does not fit shared memory");
  fused_geom(G, L, qout, H, *tb, fg);
  return FLPR_OK;
}

}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_lpr2d_fused_supported(const int* h_G, const int* h_L, const int* h_qout, int H, int order,
                               int C) {
  FusedTables tb;
  FusedGeom fg;
  return fused2d_check(h_G, h_L, h_qout, H, order, C, &tb, &fg) == FLPR_OK ? 1 : 0;
}

size_t flpr_lpr2d_fused_ws(const int* h_G, const int* h_L, const int* h_qout, int H, int order,
                           int C) {
  FusedTables tb;
  FusedGeom fg;
  if (fused2d_check(h_G, h_L, h_qout, H, order, C, &tb, &fg) != FLPR_OK) return 0;
  ArenaSize ar;
  ar.take<float2>((size_t)(1 + C) * fg.L1h * fg.L0);
  ar.take<float2>(fg.w_elems);
  ar.take<float2>(2 * (size_t)fg.L0);
  ar.take<float2>(2 * (size_t)fg.L1);
  ar.take<double>((size_t)H * fg.M * tb.nt);
  return ar.used;
}

int flpr_lpr2d_fused(const int* h_G, const int* h_L, const int* h_qout, int H, int npow, int order,
                     int C, int ny, const void* d_spec, const void* d_F, double scale,
                     const double* d_Q, double reg, float* d_S, double* d_my, double* d_dots,
                     double* d_scalar, void* d_ws, size_t ws_bytes, void* stream) {
  FusedTables tb;
  FusedGeom fg;
  FLPR_TRY(fused2d_check(h_G, h_L, h_qout, H, order, C, &tb, &fg));
  FLPR_CHECK_ARG(ny >= 0 && ny <= C, "fused2d: ny=%d", ny);
  FLPR_CHECK_ARG(npow >= 2 * order + 1, "fused2d: npow=%d < 2*order+1", npow);
  if (ws_bytes < flpr_lpr2d_fused_ws(h_G, h_L, h_qout, H, order, C)) {
    set_error("fused2d: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  Arena ar(d_ws, ws_bytes);
  float2* Yt = ar.take<float2>((size_t)(1 + C) * fg.L1h * fg.L0);
  float2* W = ar.take<float2>(fg.w_elems);
  float2* tw0 = ar.take<float2>(2 * (size_t)fg.L0);
  float2* tw1 = ar.take<float2>(2 * (size_t)fg.L1);
  double* zbuf = ar.take<double>((size_t)H * fg.M * tb.nt);
  float2* tw20 = tw0 + fg.L0;
  float2* tw21 = tw1 + fg.L1;
  cudaStream_t s = as_stream(stream);
  const float2* spec = static_cast<const float2*>(d_spec);
  const double2* F = static_cast<const double2*>(d_F);
  switch (fg.L0 / 32) {
#define FLPR_E0(V)                                                                              \
  case V:                                                                                       \
    return dispatch_e1<V>(fg.L1 / 32, tb, fg, H, npow, order, C, ny, spec, F, scale, d_Q, reg,  \
                          d_S, d_my, d_dots, d_scalar, Yt, W, tw0, tw20, tw1, tw21, zbuf, s);
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

}  // extern "C"
