// Bandwidth-proposal MLP: BF16-in / FP32-accumulate training and inference.
//
// The network is a plain stack of dense layers, h_{l+1} = relu(h_l W_l^T + b_l)
// (no ReLU after the last layer), with W_l stored (out, in) row-major.  All
// products go through one tiled tensor-core GEMM: 64 x 64 output tiles per
// 128-thread block, 32-deep K steps staged in shared memory, warp tiles of
// 32 x 32 built from mma.sync m16n8k16 (BF16 operands, FP32 accumulators).
// At the widths used here (<= 512) a GEMM launch is latency-bound, so one
// simple tile shape serves forward, backward and weight-gradient products;
// the epilogue fuses the bias, the ReLU, the ReLU-derivative mask and the
// FP32 / BF16 stores.  Master weights and Adam moments stay in FP32.
#include <cuda_bf16.h>

#include "common.cuh"

namespace flpr {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32;
constexpr int kGemmThreads = 128;
constexpr int kPad = 8;  // bf16 elements of padding per shared row (conflict-free fragment loads)

// Element (m, k) of A and (k, n) of B under the four storage orders.
//   A: a_trans = 0 -> A[m * lda + k];  1 -> A[k * lda + m]
//   B: b_nk    = 0 -> B[k * ldb + n];  1 -> B[n * ldb + k]   (W_l as stored)
struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16* A;
  int lda, a_trans;
  const __nv_bfloat16* B;
  int ldb, b_nk;
  const float* bias;           // (N) or null
  int relu;                    // apply max(0, .) after the bias
  const __nv_bfloat16* mask;   // multiply by (mask[m * ldm + n] > 0) or null
  int ldm;
  float* C32;                  // (M, N) fp32 output or null
  __nv_bfloat16* C16;          // (M, N) bf16 output or null
  int ldc;
};

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(kGemmThreads)
gemm_bf16_kernel(GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 As[kBM][kBK + kPad];  // (m, k)
  __shared__ __align__(16) __nv_bfloat16 Bs[kBN][kBK + kPad];  // (n, k)
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int grp = lane >> 2, tig = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0f;
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  for (int k0 = 0; k0 < g.K; k0 += kBK) {
    for (int i = threadIdx.x; i < kBM * kBK; i += kGemmThreads) {
      // consecutive threads walk the contiguous index of each operand
      int m, k;
      if (g.a_trans) {
        m = i % kBM;
        k = i / kBM;
      } else {
        k = i % kBK;
        m = i / kBK;
      }
      const int gm = m0 + m, gk = k0 + k;
      __nv_bfloat16 v = zero;
      if (gm < g.M && gk < g.K)
        v = g.a_trans ? g.A[(size_t)gk * g.lda + gm] : g.A[(size_t)gm * g.lda + gk];
      As[m][k] = v;
    }
    for (int i = threadIdx.x; i < kBN * kBK; i += kGemmThreads) {
      int n, k;
      if (g.b_nk) {
        k = i % kBK;
        n = i / kBK;
      } else {
        n = i % kBN;
        k = i / kBN;
      }
      const int gn = n0 + n, gk = k0 + k;
      __nv_bfloat16 v = zero;
      if (gn < g.N && gk < g.K)
        v = g.b_nk ? g.B[(size_t)gn * g.ldb + gk] : g.B[(size_t)gk * g.ldb + gn];
      Bs[n][k] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + grp;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tig]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tig]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tig + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tig + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = wn + j * 8 + grp;
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * tig]);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * tig + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
  // epilogue: accumulator e of tile (i, j) is row grp (+8 for e >= 2), column 2 tig + (e & 1)
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + i * 16 + grp + (e >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * tig + (e & 1);
        if (m >= g.M || n >= g.N) continue;
        float v = acc[i][j][e];
        if (g.bias) v += g.bias[n];
        if (g.relu) v = fmaxf(v, 0.0f);
        if (g.mask && !(__bfloat162float(g.mask[(size_t)m * g.ldm + n]) > 0.0f)) v = 0.0f;
        if (g.C32) g.C32[(size_t)m * g.ldc + n] = v;
        if (g.C16) g.C16[(size_t)m * g.ldc + n] = __float2bfloat16(v);
      }
}

// out[n] = sum_m X[m * ldx + n], fixed summation order.
__global__ void colsum_kernel(int M, int N, const float* __restrict__ X, int ldx,
                              float* __restrict__ out) {
  const int n = blockIdx.x;
  __shared__ float sh[256];
  float s = 0.0f;
  for (int m = threadIdx.x; m < M; m += blockDim.x) s += X[(size_t)m * ldx + n];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = sh[0];
}

// Mean-squared error over B outputs and its gradient: dy = 2 (y - t) / B.
__global__ void mse_kernel(int B, const float* __restrict__ y, const float* __restrict__ t,
                           float* __restrict__ dy, float* __restrict__ loss) {
  __shared__ float sh[256];
  float s = 0.0f;
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    const float e = y[i] - t[i];
    dy[i] = 2.0f * e / (float)B;
    s += e * e;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[0] = sh[0] / (float)B;
}

// Adam on FP32 master parameters; refreshes the BF16 copy.
__global__ void adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ grad,
                            float* __restrict__ m, float* __restrict__ v,
                            __nv_bfloat16* __restrict__ p16, float lr, float b1, float b2,
                            float eps, float wd, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = grad[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (p16) p16[i] = __float2bfloat16(pi);
  }
}

__global__ void f32_to_bf16_kernel(int64_t n, const float* __restrict__ x,
                                   __nv_bfloat16* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

int launch_gemm(const GemmArgs& g, cudaStream_t s) {
  FLPR_CHECK_ARG(g.M >= 1 && g.N >= 1 && g.K >= 1, "mlp_gemm: M=%d N=%d K=%d", g.M, g.N, g.K);
  FLPR_CHECK_ARG(g.A && g.B && (g.C32 || g.C16), "mlp_gemm: null operand");
  FLPR_CHECK_ARG(g.lda >= (g.a_trans ? g.M : g.K) && g.ldb >= (g.b_nk ? g.K : g.N) && g.ldc >= g.N,
                 "mlp_gemm: leading dimensions");
  FLPR_CHECK_ARG(!g.mask || g.ldm >= g.N, "mlp_gemm: mask leading dimension");
  dim3 grid((g.N + kBN - 1) / kBN, (g.M + kBM - 1) / kBM);
  FLPR_CHECK_ARG(grid.y <= 65535, "mlp_gemm: M=%d too large", g.M);
  gemm_bf16_kernel<<<grid, kGemmThreads, 0, s>>>(g);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int launch_colsum(int M, int N, const float* X, int ldx, float* out, cudaStream_t s) {
  colsum_kernel<<<N, 256, 0, s>>>(M, N, X, ldx, out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

constexpr int kMaxLayers = 8;

// Packed parameter layout of a network with dims[0..nl]: for each layer l,
// W_l (dims[l+1] x dims[l]) then b_l (dims[l+1]); bf16 copies use the same
// offsets.
int64_t param_offsets(int nl, const int* dims, int64_t* w_off, int64_t* b_off) {
  int64_t o = 0;
  for (int l = 0; l < nl; ++l) {
    w_off[l] = o;
    o += (int64_t)dims[l + 1] * dims[l];
    b_off[l] = o;
    o += dims[l + 1];
  }
  return o;
}

int check_dims(int nl, const int* dims) {
  FLPR_CHECK_ARG(nl >= 1 && nl <= kMaxLayers, "mlp: %d layers (1..%d)", nl, kMaxLayers);
  for (int l = 0; l <= nl; ++l)
    FLPR_CHECK_ARG(dims[l] >= 1 && dims[l] <= 4096, "mlp: dims[%d]=%d", l, dims[l]);
  return FLPR_OK;
}

// Activation workspace: for each layer l < nl - 1 the bf16 output h_{l+1}
// (B x dims[l+1]); then fp32 and bf16 gradient buffers of the widest layer.
struct ActLayout {
  int64_t h_off[kMaxLayers];
  int64_t gz32_a, gz32_b, gz16_a, gz16_b;  // byte offsets
  size_t bytes;
};

ActLayout act_layout(int nl, const int* dims, int B) {
  ActLayout a;
  size_t o = 0;
  int wmax = 1;
  for (int l = 0; l <= nl; ++l) wmax = dims[l] > wmax ? dims[l] : wmax;
  for (int l = 0; l < nl - 1; ++l) {
    a.h_off[l] = (int64_t)o;
    o = align_up(o + sizeof(__nv_bfloat16) * (size_t)B * dims[l + 1]);
  }
  const size_t f = sizeof(float) * (size_t)B * wmax, h = sizeof(__nv_bfloat16) * (size_t)B * wmax;
  a.gz32_a = (int64_t)o;
  o = align_up(o + f);
  a.gz32_b = (int64_t)o;
  o = align_up(o + f);
  a.gz16_a = (int64_t)o;
  o = align_up(o + h);
  a.gz16_b = (int64_t)o;
  o = align_up(o + h);
  a.bytes = o;
  return a;
}

}  // namespace
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_mlp_gemm(int M, int N, int K, const void* d_A, int lda, int a_trans, const void* d_B,
                  int ldb, int b_nk, const float* d_bias, int relu, const void* d_mask, int ldm,
                  float* d_C32, void* d_C16, int ldc, void* stream) {
  GemmArgs g;
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = static_cast<const __nv_bfloat16*>(d_A);
  g.lda = lda;
  g.a_trans = a_trans ? 1 : 0;
  g.B = static_cast<const __nv_bfloat16*>(d_B);
  g.ldb = ldb;
  g.b_nk = b_nk ? 1 : 0;
  g.bias = d_bias;
  g.relu = relu ? 1 : 0;
  g.mask = static_cast<const __nv_bfloat16*>(d_mask);
  g.ldm = ldm;
  g.C32 = d_C32;
  g.C16 = static_cast<__nv_bfloat16*>(d_C16);
  g.ldc = ldc;
  return launch_gemm(g, as_stream(stream));
}

int64_t flpr_mlp_param_count(int nlayers, const int* h_dims) {
  if (check_dims(nlayers, h_dims) != FLPR_OK) return -1;
  int64_t w[kMaxLayers], b[kMaxLayers];
  return param_offsets(nlayers, h_dims, w, b);
}

size_t flpr_mlp_ws(int nlayers, const int* h_dims, int batch) {
  if (check_dims(nlayers, h_dims) != FLPR_OK || batch < 1) return 0;
  return act_layout(nlayers, h_dims, batch).bytes;
}

int flpr_mlp_fwd(int nlayers, const int* h_dims, const void* d_params16, const float* d_params32,
                 int batch, const void* d_x16, float* d_out, void* d_ws, size_t ws_bytes,
                 void* stream) {
  FLPR_TRY(check_dims(nlayers, h_dims));
  FLPR_CHECK_ARG(batch >= 1, "mlp_fwd: batch=%d", batch);
  const ActLayout al = act_layout(nlayers, h_dims, batch);
  if (ws_bytes < al.bytes) {
    set_error("mlp_fwd: workspace too small (%zu < %zu)", ws_bytes, al.bytes);
    return FLPR_ERR_WORKSPACE;
  }
  int64_t wo[kMaxLayers], bo[kMaxLayers];
  param_offsets(nlayers, h_dims, wo, bo);
  const __nv_bfloat16* p16 = static_cast<const __nv_bfloat16*>(d_params16);
  char* ws = static_cast<char*>(d_ws);
  const __nv_bfloat16* in = static_cast<const __nv_bfloat16*>(d_x16);
  for (int l = 0; l < nlayers; ++l) {
    const bool last = l == nlayers - 1;
    GemmArgs g;
    memset(&g, 0, sizeof(g));
    g.M = batch;
    g.N = h_dims[l + 1];
    g.K = h_dims[l];
    g.A = in;
    g.lda = h_dims[l];
    g.B = p16 + wo[l];
    g.ldb = h_dims[l];
    g.b_nk = 1;
    g.bias = d_params32 + bo[l];
    g.relu = last ? 0 : 1;
    g.ldc = h_dims[l + 1];
    if (last) {
      g.C32 = d_out;
    } else {
      g.C16 = reinterpret_cast<__nv_bfloat16*>(ws + al.h_off[l]);
    }
    FLPR_TRY(launch_gemm(g, as_stream(stream)));
    if (!last) in = g.C16;
  }
  return FLPR_OK;
}

int flpr_mlp_bwd(int nlayers, const int* h_dims, const void* d_params16, int batch,
                 const void* d_x16, const float* d_dout, float* d_grad32, void* d_ws,
                 size_t ws_bytes, void* stream) {
  FLPR_TRY(check_dims(nlayers, h_dims));
  FLPR_CHECK_ARG(batch >= 1, "mlp_bwd: batch=%d", batch);
  const ActLayout al = act_layout(nlayers, h_dims, batch);
  if (ws_bytes < al.bytes) {
    set_error("mlp_bwd: workspace too small (%zu < %zu)", ws_bytes, al.bytes);
    return FLPR_ERR_WORKSPACE;
  }
  cudaStream_t s = as_stream(stream);
  int64_t wo[kMaxLayers], bo[kMaxLayers];
  param_offsets(nlayers, h_dims, wo, bo);
  const __nv_bfloat16* p16 = static_cast<const __nv_bfloat16*>(d_params16);
  char* ws = static_cast<char*>(d_ws);
  float* gz32[2] = {reinterpret_cast<float*>(ws + al.gz32_a), reinterpret_cast<float*>(ws + al.gz32_b)};
  __nv_bfloat16* gz16[2] = {reinterpret_cast<__nv_bfloat16*>(ws + al.gz16_a),
                            reinterpret_cast<__nv_bfloat16*>(ws + al.gz16_b)};
  // dz of the last layer = d_dout (batch x dims[nl])
  const int nout = h_dims[nlayers];
  {
    int nb = (int)(((int64_t)batch * nout + 255) / 256);
    if (nb > 4096) nb = 4096;
    f32_to_bf16_kernel<<<nb, 256, 0, s>>>((int64_t)batch * nout, d_dout, gz16[0]);
    FLPR_LAUNCH_CHECK();
  }
  const float* dz32 = d_dout;
  int cur = 0;
  for (int l = nlayers - 1; l >= 0; --l) {
    const __nv_bfloat16* hin =
        l == 0 ? static_cast<const __nv_bfloat16*>(d_x16)
               : reinterpret_cast<const __nv_bfloat16*>(ws + al.h_off[l - 1]);
    // dW_l = dz^T h_l  (dims[l+1] x dims[l]);  db_l = column sums of dz
    GemmArgs g;
    memset(&g, 0, sizeof(g));
    g.M = h_dims[l + 1];
    g.N = h_dims[l];
    g.K = batch;
    g.A = gz16[cur];
    g.lda = h_dims[l + 1];
    g.a_trans = 1;
    g.B = hin;
    g.ldb = h_dims[l];
    g.b_nk = 0;
    g.C32 = d_grad32 + wo[l];
    g.ldc = h_dims[l];
    FLPR_TRY(launch_gemm(g, s));
    FLPR_TRY(launch_colsum(batch, h_dims[l + 1], dz32, h_dims[l + 1], d_grad32 + bo[l], s));
    if (l == 0) break;
    // dz_{l-1} = (dz W_l) * (h_l > 0)
    GemmArgs gb;
    memset(&gb, 0, sizeof(gb));
    gb.M = batch;
    gb.N = h_dims[l];
    gb.K = h_dims[l + 1];
    gb.A = gz16[cur];
    gb.lda = h_dims[l + 1];
    gb.B = p16 + wo[l];
    gb.ldb = h_dims[l];
    gb.b_nk = 0;
    gb.mask = hin;
    gb.ldm = h_dims[l];
    gb.C32 = gz32[1 - cur];
    gb.C16 = gz16[1 - cur];
    gb.ldc = h_dims[l];
    FLPR_TRY(launch_gemm(gb, s));
    cur = 1 - cur;
    dz32 = gz32[cur];
  }
  return FLPR_OK;
}

int flpr_mlp_step(int64_t nparams, float* d_params32, void* d_params16, const float* d_grad32,
                  float* d_m, float* d_v, float lr, float beta1, float beta2, float eps,
                  float weight_decay, int step, void* stream) {
  FLPR_CHECK_ARG(nparams >= 1 && step >= 1, "mlp_step: n=%lld step=%d", (long long)nparams, step);
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  int nb = (int)((nparams + 255) / 256);
  if (nb > 8 * sm_count()) nb = 8 * sm_count();
  adam_kernel<<<nb, 256, 0, as_stream(stream)>>>(nparams, d_params32, d_grad32, d_m, d_v,
                                                  static_cast<__nv_bfloat16*>(d_params16), lr,
                                                  beta1, beta2, eps, weight_decay, c1, c2);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_mlp_mse(int batch, const float* d_y, const float* d_t, float* d_dy, float* d_loss,
                 void* stream) {
  FLPR_CHECK_ARG(batch >= 1, "mlp_mse: batch=%d", batch);
  mse_kernel<<<1, 256, 0, as_stream(stream)>>>(batch, d_y, d_t, d_dy, d_loss);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_to_bf16(int64_t n, const float* d_x, void* d_y, void* stream) {
  FLPR_CHECK_ARG(n >= 1, "to_bf16: n=%lld", (long long)n);
  int nb = (int)((n + 255) / 256);
  if (nb > 8 * sm_count()) nb = 8 * sm_count();
  f32_to_bf16_kernel<<<nb, 256, 0, as_stream(stream)>>>(n, d_x, static_cast<__nv_bfloat16*>(d_y));
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
