// Fused inference of the bandwidth-proposal network on the fifth-generation
// tensor cores (tcgen05, sm_100a).
//
// The network h_{l+1} = relu(h_l W_l^T + b_l) with hidden width 256 and one
// output runs in ONE launch: a CTA of four warps takes 128 rows of the batch
// (the UMMA M), keeps their activations in shared memory as the A operand of
// the next layer (BF16, K-major, 128-byte swizzle) and accumulates every
// layer's 128 x 256 product in tensor memory (256 FP32 columns).  Weights
// stream through a ring of three 64-deep K chunks (256 rows x 128 bytes
// each) loaded with cp.async; one elected thread issues the tcgen05.mma
// instructions (M = 128, N = 256, K = 16, BF16 x BF16 -> FP32) and commits
// them to a per-stage mbarrier.  The epilogue of each layer reads the
// accumulator with tcgen05.ld (each warp its 32 TMEM lanes = rows), adds the
// FP32 bias, applies the ReLU and rounds to BF16 into the next A operand;
// the last layer (one output) is a dot product of the last hidden row with
// the output weights in registers.  Every wait on an mbarrier is bounded:
// on expiry the CTA records FLPR_ERR_TIMEOUT in the status word, waits for
// its own copies, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "common.cuh"

namespace flpr {
namespace {

constexpr int kTM = 128;                 // batch rows per CTA (UMMA M)
constexpr int kHid = 256;                // hidden width (UMMA N)
constexpr int kKC = 64;                  // K elements per chunk: one 128-byte swizzle row
constexpr int kMaxInChunks = 7;          // input width <= 448
constexpr int kStages = 3;               // weight chunk ring
constexpr int kThreads = 128;            // four warps: one per 32 TMEM lanes
constexpr int kMaxLayersTc = 8;
constexpr int kAChunk = kTM * 128;       // 16 KB
constexpr int kBChunk = kHid * 128;      // 32 KB
constexpr uint32_t kSpinLimit = 1u << 24;
constexpr uint32_t kTmemCols = 256;

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 256, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            ((uint32_t)(kHid >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);

struct TcArgs {
  int nlayers;
  int dims[kMaxLayersTc + 1];
  int64_t w_off[kMaxLayersTc];   // BF16 element offsets of W_l in the packed parameters
  int64_t b_off[kMaxLayersTc];   // FP32 element offsets of b_l
  int nchunks[kMaxLayersTc];     // K chunks of each hidden layer
  int total_chunks;
  int batch;
  const __nv_bfloat16* p16;
  const float* p32;
  const __nv_bfloat16* x16;
  float* out;
  int* status;
};

// byte offset of (row, 16-byte column c16) in a K-major 128-byte-swizzled
// tile: 8-row groups 1024 bytes apart, the 16-byte column XORed with row % 8
__device__ __forceinline__ uint32_t sw128(int row, int c16) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((c16 ^ (row & 7)) << 4));
}

// shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand
// starting at shared address saddr (1024-aligned atom base plus a 32-byte
// step per K = 16 slice): stride between 8-row groups 1024 bytes, version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;                   // leading byte offset (16 B; unused when swizzled)
  d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset
  d |= (uint64_t)1 << 46;                   // descriptor version
  d |= (uint64_t)2 << 61;                   // 128-byte swizzle
  return d;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_pending(int n) {
  // wait until at most n groups of this thread are pending (n < kStages)
  switch (n) {
    case 0: asm volatile("cp.async.wait_group 0;\n" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;\n" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 2;\n" ::: "memory"); break;
  }
}
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// bounded wait for the given phase parity of an mbarrier
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                          uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z),
      "r"(z)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// the global chunk sequence: layer of chunk j and its K index within the layer
__device__ __forceinline__ void chunk_of(const TcArgs& a, int j, int* layer, int* kc) {
  int l = 0;
  while (j >= a.nchunks[l]) {
    j -= a.nchunks[l];
    ++l;
  }
  *layer = l;
  *kc = j;
}

// issue the cp.async copies of weight chunk j into ring stage s (rows of
// W_l beyond its K are zero-filled)
__device__ __forceinline__ void load_w_chunk(const TcArgs& a, int j, uint32_t sB) {
  int l, kc;
  chunk_of(a, j, &l, &kc);
  const int K = a.dims[l];
  const __nv_bfloat16* W = a.p16 + a.w_off[l];
  for (int v = threadIdx.x; v < kHid * 8; v += kThreads) {
    const int n = v >> 3, c16 = v & 7;
    const int k = kc * kKC + c16 * 8;
    const int bytes = k < K ? 16 : 0;   // K is a multiple of 8
    cp_async16(sB + sw128(n, c16), bytes ? (const void*)(W + (int64_t)n * K + k) : (const void*)W,
               bytes);
  }
}

__global__ void __launch_bounds__(kThreads, 1) mlp_infer_tc_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-aligned operand region: A chunks, then the B ring
  const uint32_t base_u32 = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (base_u32 & 1023u)) & 1023u;
  unsigned char* smem = smem_raw + pad;
  const uint32_t sA = base_u32 + pad;
  const uint32_t sB = sA + kMaxInChunks * kAChunk;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kMaxInChunks * kAChunk + kStages * kBChunk);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kStages);
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * kTM;
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // input rows of this CTA (zero beyond the batch and beyond K0), with the
  // first weight chunk, as the first copy group
  {
    const int K0 = a.dims[0];
    const int nc0 = a.nchunks[0];
    for (int v = threadIdx.x; v < kTM * nc0 * 8; v += kThreads) {
      const int kc = v / (kTM * 8), r = v % (kTM * 8);
      const int m = r >> 3, c16 = r & 7;
      const int k = kc * kKC + c16 * 8;
      const int gm = row0 + m;
      const int bytes = (gm < a.batch && k < K0) ? 16 : 0;
      cp_async16(sA + kc * kAChunk + sw128(m, c16),
                 bytes ? (const void*)(a.x16 + (int64_t)gm * K0 + k) : (const void*)a.x16, bytes);
    }
  }
  int issued = 0;
  for (; issued < kStages && issued < a.total_chunks; ++issued) {
    load_w_chunk(a, issued, sB + (issued % kStages) * kBChunk);
    cp_async_commit();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  uint32_t phase[kStages] = {0u, 0u, 0u};
  float acc_out = 0.0f;   // last-layer output of this thread's row

  for (int j = 0; j < a.total_chunks; ++j) {
    const int s = j % kStages;
    int l, kc;
    chunk_of(a, j, &l, &kc);
    // chunk j (and, for j = 0, the input) has landed: this thread's copies,
    // then everyone's through the barrier; the proxy fence makes the
    // generic-proxy writes visible to the tensor core's reads
    cp_async_wait_pending(issued - j - 1);
    fence_async_shared();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
#pragma unroll
      for (int kk = 0; kk < kKC / 16; ++kk) {
        const uint64_t da = umma_desc(sA + kc * kAChunk + kk * 32);
        const uint64_t db = umma_desc(sB + s * kBChunk + kk * 32);
        umma_bf16(tmem, da, db, (kc > 0 || kk > 0) ? 1u : 0u);
      }
      umma_commit(&bars[s]);
    }
    // the products of chunk j are done: stage s is free and, after the
    // layer's last chunk, the accumulator is complete
    if (!mbar_wait(&bars[s], phase[s])) s_abort = 1;
    phase[s] ^= 1u;
    __syncthreads();
    if (s_abort) break;
    tc_fence_after();
    if (kc == a.nchunks[l] - 1) {
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
      const int m = warp * 32 + lane;
      const float* bias = a.p32 + a.b_off[l];
      const bool last_hidden = (l == a.nlayers - 2);
      if (last_hidden) acc_out = a.p32[a.b_off[l + 1]];
      const __nv_bfloat16* wout = a.p16 + a.w_off[a.nlayers - 1];
      for (int c0 = 0; c0 < kHid; c0 += 16) {
        float v[16];
        tmem_ld16(trow + (uint32_t)c0, v);
        __align__(16) __nv_bfloat16 h[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) h[i] = __float2bfloat16_rn(fmaxf(v[i] + bias[c0 + i], 0.0f));
        if (last_hidden) {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            acc_out += __bfloat162float(h[i]) * __bfloat162float(wout[c0 + i]);
        } else {
          // next layer's A operand: K index c0..c0+15 of row m
          const int kcn = c0 / kKC, c16 = (c0 % kKC) / 8;
          unsigned char* dst = smem + kcn * kAChunk;
          *reinterpret_cast<uint4*>(dst + sw128(m, c16)) = *reinterpret_cast<const uint4*>(h);
          *reinterpret_cast<uint4*>(dst + sw128(m, c16 + 1)) =
              *reinterpret_cast<const uint4*>(h + 8);
        }
      }
      tc_fence_before();
    }
    // refill stage s with chunk j + kStages
    if (issued < a.total_chunks) {
      load_w_chunk(a, issued, sB + (issued % kStages) * kBChunk);
      ++issued;
    }
    cp_async_commit();   // (an empty group keeps the pending count uniform)
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  tc_fence_before();
  __syncthreads();
  if (!s_abort) {
    const int gm = row0 + warp * 32 + lane;
    if (gm < a.batch) a.out[gm] = acc_out;
  } else if (threadIdx.x == 0 && a.status != nullptr) {
    atomicExch(a.status, FLPR_ERR_TIMEOUT);
  }
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

constexpr size_t kTcSmem = (size_t)kMaxInChunks * kAChunk + (size_t)kStages * kBChunk +
                           1024 /* alignment */ + kStages * sizeof(uint64_t) + 16;

}  // namespace
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_mlp_infer_supported(int nlayers, const int* h_dims) {
  if (nlayers < 2 || nlayers > kMaxLayersTc || h_dims == nullptr) return 0;
  if (h_dims[0] < 1 || h_dims[0] > kMaxInChunks * kKC || h_dims[0] % 8 != 0) return 0;
  for (int l = 1; l < nlayers; ++l)
    if (h_dims[l] != kHid) return 0;
  return h_dims[nlayers] == 1 ? 1 : 0;
}

int flpr_mlp_infer(int nlayers, const int* h_dims, const void* d_params16,
                   const float* d_params32, int batch, const void* d_x16, float* d_out,
                   int* d_status, void* stream) {
  FLPR_CHECK_ARG(flpr_mlp_infer_supported(nlayers, h_dims) == 1,
                 "mlp_infer: needs input width <= 448 (multiple of 8), hidden widths 256, one "
                 "output");
  FLPR_CHECK_ARG(batch >= 1, "mlp_infer: batch=%d", batch);
  FLPR_CHECK_ARG(d_params16 && d_params32 && d_x16 && d_out, "mlp_infer: null pointer");
  TcArgs a;
  memset(&a, 0, sizeof(a));
  a.nlayers = nlayers;
  int64_t off = 0;
  for (int l = 0; l <= nlayers; ++l) a.dims[l] = h_dims[l];
  for (int l = 0; l < nlayers; ++l) {
    a.w_off[l] = off;
    off += (int64_t)h_dims[l] * h_dims[l + 1];
    a.b_off[l] = off;
    off += h_dims[l + 1];
    // the operand copies move 16-byte vectors of the weight rows
    FLPR_CHECK_ARG(((uintptr_t)d_params16 + 2 * (uintptr_t)a.w_off[l]) % 16 == 0,
                   "mlp_infer: weights of layer %d not 16-byte aligned", l);
  }
  FLPR_CHECK_ARG((uintptr_t)d_x16 % 16 == 0, "mlp_infer: inputs not 16-byte aligned");
  a.total_chunks = 0;
  for (int l = 0; l < nlayers - 1; ++l) {
    a.nchunks[l] = (h_dims[l] + kKC - 1) / kKC;
    a.total_chunks += a.nchunks[l];
  }
  a.batch = batch;
  a.p16 = static_cast<const __nv_bfloat16*>(d_params16);
  a.p32 = d_params32;
  a.x16 = static_cast<const __nv_bfloat16*>(d_x16);
  a.out = d_out;
  a.status = d_status;
  FLPR_CUDA(cudaFuncSetAttribute(mlp_infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTcSmem));
  const int grid = (batch + kTM - 1) / kTM;
  mlp_infer_tc_kernel<<<grid, kThreads, kTcSmem, as_stream(stream)>>>(a);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
