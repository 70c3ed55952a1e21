// Fused inference of the bandwidth-proposal network on the fifth-generation
// tensor cores (tcgen05, sm_100a).
//
// The network h_{l+1} = relu(h_l W_l^T + b_l) with hidden width 256 and one
// output runs in ONE launch: a CTA takes 128 rows of the batch (the UMMA M),
// keeps their activations in shared memory as the A operand of the next
// layer (BF16, K-major, 128-byte swizzle) and accumulates each layer's
// 128 x 256 product in tensor memory, alternating between two 256-column
// accumulators so that a layer's products can start while the previous
// layer's epilogue is still reading its own.  The CTA is warp specialised:
//   - warp 8 (one lane) issues the tensor-map copies (cp.async.bulk.tensor,
//     128-byte swizzle: the copy engine writes the UMMA operand layout
//     itself, columns beyond K read as zero): the input chunks (64 columns
//     of the CTA's rows, each on its own barrier, the box only as tall as a
//     batch smaller than the tile) beside the weights, which stream through
//     a ring of three 64-deep K chunks (256 rows x 128 bytes);
//   - warp 9 (one lane) issues the tcgen05.mma instructions (M = 128,
//     N = 256, K = 16, BF16 x BF16 -> FP32) for a K chunk as soon as its
//     weights and its 64 A columns are there, committing each chunk to its
//     stage's "empty" barrier (the producer refills the stage after it) and
//     each layer's last chunk to the accumulator barrier;
//   - warps 0-7 run each layer's epilogue, warp w on TMEM lanes
//     32 (w % 4) .. + 31 (its rows) and columns 128 (w / 4) .. + 127:
//     tcgen05.ld of the accumulator, FP32 bias (cached in shared memory) on
//     the packed two-lane adds, rounding to BF16 pairs and ReLU into the
//     next layer's A operand, one arrival per 64 columns on the barrier the
//     next layer's products on those K columns wait for; the last layer (one
//     output) is a dot product of the last hidden row with the output
//     weights on packed two-lane FMAs, the two column halves added in shared
//     memory.
// Every wait on an mbarrier is bounded: on expiry the CTA records
// FLPR_ERR_TIMEOUT in the status word, the producer waits (bounded) for its
// copies in flight, the MMA issuer for its products, and the tensor memory
// is freed before the CTA returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include "common.cuh"

namespace flpr {
namespace {

constexpr int kTM = 128;                 // batch rows per CTA (UMMA M)
constexpr int kHid = 256;                // hidden width (UMMA N)
constexpr int kKC = 64;                  // K elements per chunk: one 128-byte swizzle row
constexpr int kMaxInChunks = 7;          // input width <= 448
constexpr int kStages = 3;               // weight chunk ring
constexpr int kEpiWarps = 8;             // warps 0-7: TMEM lanes 32 (w % 4) ..., columns half w / 4
constexpr int kProdWarp = 8;             // tensor-map copies
constexpr int kMmaWarp = 9;              // tcgen05.mma issue
constexpr int kThreads = 32 * 10;
constexpr int kMaxLayersTc = 8;
constexpr int kAChunk = kTM * 128;       // 16 KB
constexpr int kBChunk = kHid * 128;      // 32 KB
constexpr uint32_t kSpinLimit = 1u << 24;
constexpr int kHidChunks = kHid / kKC;   // 64-wide chunks of a hidden layer
constexpr uint32_t kTmemCols = 2 * kHid;  // two accumulators: layer l uses columns (l % 2) * 256

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 256, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            ((uint32_t)(kHid >> 3) << 17) | ((uint32_t)(kTM >> 4) << 24);

struct TcArgs {
  CUtensorMap tm_w[kMaxLayersTc];  // W_l (K_l columns x 256 rows), boxes of 64 x 256
  CUtensorMap tm_x;                // inputs (K_0 columns x batch rows), boxes of 64 x 128
  int nlayers;
  int dims[kMaxLayersTc + 1];
  int64_t w_off[kMaxLayersTc];     // BF16 element offsets of W_l in the packed parameters
  int64_t b_off[kMaxLayersTc];     // FP32 element offsets of b_l
  int nchunks[kMaxLayersTc];       // K chunks of each hidden layer
  int total_chunks;
  int batch;
  int in_box_rows;                 // rows of each input box (the batch rounded up to 8, <= 128)
  const __nv_bfloat16* p16;
  const float* p32;
  float* out;
  int* status;
};

// byte offset of (row, 16-byte column c16) in a K-major 128-byte-swizzled
// tile: 8-row groups 1024 bytes apart, the 16-byte column XORed with row % 8
// (the layout the tensor-map copies with 128-byte swizzle write)
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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// bounded wait for the given phase parity of an mbarrier; gives up early
// when another role of the CTA has given up (abort flag; null for the
// drains of copies and products in flight, which run to the bound)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          const volatile int* abort_flag) {
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
    if (abort_flag != nullptr && (it & 1023u) == 1023u && *abort_flag) return false;
  }
  return false;
}

// 2-D tensor-map copy of one box into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* tm, int c0, int c1,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
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

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane (no
// wait: the caller issues tcgen05.wait::ld before using them)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// FP32 pairs in one 64-bit register for the packed two-lane instructions
// (each lane rounded as the scalar instruction)
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}

// relu(bf16(acc + bias)) of two adjacent columns as one BF16 pair, the
// lower column in the low half: the sums on add.rn.f32x2, both roundings
// to BF16 (nearest even) in one conversion, the ReLU on the pair (the same
// values as rounding after the ReLU, up to the sign of a zero)
__device__ __forceinline__ uint32_t bias_relu_bf16x2(uint32_t a0, uint32_t a1, float b0,
                                                     float b1) {
  unsigned long long sum;
  asm("add.rn.f32x2 %0, %1, %2;"
      : "=l"(sum)
      : "l"(f2_pack(__uint_as_float(a0), __uint_as_float(a1))), "l"(f2_pack(b0, b1)));
  const float2 v = f2_unpack(sum);
  __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
  h = __hmax2(h, __float2bfloat162_rn(0.0f));
  return *reinterpret_cast<uint32_t*>(&h);
}

// acc (two FP32 lanes) += h * w on fma.rn.f32x2, the BF16 pair h widened
// exactly to FP32
__device__ __forceinline__ unsigned long long fma_bf16x2(uint32_t h, float w0, float w1,
                                                         unsigned long long acc) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(d)
      : "l"(f2_pack(__uint_as_float(h << 16), __uint_as_float(h & 0xffff0000u))),
        "l"(f2_pack(w0, w1)), "l"(acc));
  return d;
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

__global__ void __launch_bounds__(kThreads, 1)
    mlp_infer_tc_kernel(const __grid_constant__ TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-aligned operand region: A chunks, then the B ring, then barriers
  // and the FP32 bias / output-weight cache
  const uint32_t base_u32 = smem_u32(smem_raw);
  const uint32_t pad = (1024u - (base_u32 & 1023u)) & 1023u;
  unsigned char* smem = smem_raw + pad;
  const uint32_t sA = base_u32 + pad;
  const uint32_t sB = sA + kMaxInChunks * kAChunk;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kMaxInChunks * kAChunk + kStages * kBChunk);
  uint64_t* full = bars;                       // [kStages] weight chunk landed
  uint64_t* empty = bars + kStages;            // [kStages] chunk's products done
  uint64_t* in_full = bars + 2 * kStages;      // [kMaxInChunks] input chunk landed
  uint64_t* acc_full = in_full + kMaxInChunks; // a layer's accumulator complete
  uint64_t* a_chunk = acc_full + 1;            // [kHidChunks] 64 activations of the next A written
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(a_chunk + kHidChunks);
  float* s_bias = reinterpret_cast<float*>(tmem_slot + 4);   // [nlayers - 1][256], 16-aligned
  float* s_wout = s_bias + (kMaxLayersTc - 1) * kHid;         // [256]
  float* s_part = s_wout + kHid;                              // [128]
  __shared__ volatile int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * kTM;
  const int nhid = a.nlayers - 1;  // layers with 256 outputs
  const int nin = a.nchunks[0];
  // the producer initialises the barriers and starts the first copies
  // (each input chunk beside the layer-0 weight chunk it meets, so the
  // first products can start when the first pair has landed) before the
  // CTA-wide set-up
  if (threadIdx.x == kProdWarp * 32) {
    s_abort = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int k = 0; k < kMaxInChunks; ++k) mbar_init(&in_full[k], 1);
    mbar_init(acc_full, 1);
    for (int c = 0; c < kHidChunks; ++c) mbar_init(&a_chunk[c], kEpiWarps * 16);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    for (int k = 0; k < nin || (k < kStages && k < a.total_chunks); ++k) {
      if (k < nin) {
        mbar_expect_tx(&in_full[k], (uint32_t)(a.in_box_rows * 128));
        tma_load_2d(sA + k * kAChunk, &a.tm_x, k * kKC, row0, &in_full[k]);
      }
      if (k < kStages && k < a.total_chunks) {
        int l, kc;
        chunk_of(a, k, &l, &kc);
        mbar_expect_tx(&full[k], (uint32_t)kBChunk);
        tma_load_2d(sB + k * kBChunk, &a.tm_w[l], kc * kKC, 0, &full[k]);
      }
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kProdWarp) {
    if (lane == 0) {
      // the rest of the weight chunks in order, each into the stage the
      // products kStages chunks earlier have released
      int issued = a.total_chunks < kStages ? a.total_chunks : kStages;
      for (int j = kStages; j < a.total_chunks; ++j) {
        const int s = j % kStages;
        if (!mbar_wait(&empty[s], (uint32_t)((j / kStages) - 1) & 1u, &s_abort)) {
          s_abort = 1;
          break;
        }
        int l, kc;
        chunk_of(a, j, &l, &kc);
        mbar_expect_tx(&full[s], (uint32_t)kBChunk);
        tma_load_2d(sB + s * kBChunk, &a.tm_w[l], kc * kKC, 0, &full[s]);
        issued = j + 1;
      }
      // the copies in flight land before the CTA can leave
      for (int j = issued - 1; j >= 0 && j >= issued - kStages; --j)
        mbar_wait(&full[j % kStages], (uint32_t)(j / kStages) & 1u, nullptr);
      for (int k = 0; k < nin; ++k) mbar_wait(&in_full[k], 0u, nullptr);
    }
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      int last = -1;
      for (int j = 0; j < a.total_chunks; ++j) {
        const int s = j % kStages;
        int l, kc;
        chunk_of(a, j, &l, &kc);
        // the chunk's A operand: an input chunk for layer 0, else the 64
        // activations of the previous layer's epilogue (which has also read
        // this layer's accumulator as it was two layers back)
        const bool a_ok = (l == 0) ? mbar_wait(&in_full[kc], 0u, &s_abort)
                                   : mbar_wait(&a_chunk[kc], (uint32_t)(l - 1) & 1u, &s_abort);
        if (!a_ok || !mbar_wait(&full[s], (uint32_t)(j / kStages) & 1u, &s_abort)) {
          s_abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t dacc = tmem + (uint32_t)((l & 1) * kHid);
#pragma unroll
        for (int kk = 0; kk < kKC / 16; ++kk) {
          const uint64_t da = umma_desc(sA + kc * kAChunk + kk * 32);
          const uint64_t db = umma_desc(sB + s * kBChunk + kk * 32);
          umma_bf16(dacc, da, db, (kc > 0 || kk > 0) ? 1u : 0u);
        }
        umma_commit(&empty[s]);
        if (kc == a.nchunks[l] - 1) umma_commit(acc_full);
        last = j;
      }
      // every product issued is complete before the tensor memory is freed
      if (last >= 0)
        mbar_wait(&empty[last % kStages], (uint32_t)(last / kStages) & 1u, nullptr);
    }
  } else {
    // epilogue warps: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows)
    // and owns columns 128 (w / 4) .. + 127 of every layer.  The bias cache
    // fills here, off the path of the first products.
    for (int i = threadIdx.x; i < nhid * kHid; i += kEpiWarps * 32) {
      const int l = i / kHid, c = i - l * kHid;
      s_bias[i] = a.p32[a.b_off[l] + c];
    }
    const __nv_bfloat16* wout = a.p16 + a.w_off[a.nlayers - 1];
    for (int c = threadIdx.x; c < kHid; c += kEpiWarps * 32) s_wout[c] = __bfloat162float(wout[c]);
    asm volatile("bar.sync 1, %0;\n" ::"n"(kEpiWarps * 32) : "memory");
    const int quarter = warp & 3, half = warp >> 2;
    const uint32_t trow = tmem + ((uint32_t)(quarter * 32) << 16);
    const int m = quarter * 32 + lane;
    float partial = 0.0f;  // this half's share of the output layer's dot product
    bool ok = true;
    for (int l = 0; l < nhid; ++l) {
      ok = __all_sync(0xffffffffu, mbar_wait(acc_full, (uint32_t)l & 1u, &s_abort));
      if (!ok) {
        s_abort = 1;
        break;
      }
      tc_fence_after();
      const float* bias = s_bias + l * kHid;
      const uint32_t tacc = trow + (uint32_t)((l & 1) * kHid);
      const bool last_hidden = (l == nhid - 1);
      // the output layer's dot product in eight independent partial sums
      unsigned long long acc2[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll 1
      for (int cc = 0; cc < kHidChunks / 2; ++cc) {
        const int c0 = (half * (kHidChunks / 2) + cc) * kKC;
        uint32_t r[4][16];
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_ld16(tacc + (uint32_t)(c0 + 16 * q), r[q]);
        tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4* b4 = reinterpret_cast<const float4*>(bias + c0 + 16 * q);
          uint32_t h2[8];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const float4 bb = b4[t];
            h2[2 * t] = bias_relu_bf16x2(r[q][4 * t], r[q][4 * t + 1], bb.x, bb.y);
            h2[2 * t + 1] = bias_relu_bf16x2(r[q][4 * t + 2], r[q][4 * t + 3], bb.z, bb.w);
          }
          if (last_hidden) {
            const float4* w4 = reinterpret_cast<const float4*>(s_wout + c0 + 16 * q);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              const float4 ww = w4[t];
              acc2[(2 * t) & 3] = fma_bf16x2(h2[2 * t], ww.x, ww.y, acc2[(2 * t) & 3]);
              acc2[(2 * t + 1) & 3] = fma_bf16x2(h2[2 * t + 1], ww.z, ww.w, acc2[(2 * t + 1) & 3]);
            }
          } else {
            // next layer's A operand: chunk c0 / 64, 16-byte columns 2q, 2q + 1
            unsigned char* dst = smem + (c0 / kKC) * kAChunk;
            *reinterpret_cast<uint4*>(dst + sw128(m, 2 * q)) =
                make_uint4(h2[0], h2[1], h2[2], h2[3]);
            *reinterpret_cast<uint4*>(dst + sw128(m, 2 * q + 1)) =
                make_uint4(h2[4], h2[5], h2[6], h2[7]);
          }
        }
        if (!last_hidden) {
          // generic-proxy writes of these 64 activations, and the
          // accumulator reads so far, ordered before the next layer's
          // products on this chunk
          fence_async_shared();
          tc_fence_before();
          mbar_arrive(&a_chunk[c0 / kKC]);
        }
      }
      if (last_hidden) {
        float2 p[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) p[i] = f2_unpack(acc2[i]);
        partial = ((p[0].x + p[0].y) + (p[1].x + p[1].y)) + ((p[2].x + p[2].y) + (p[3].x + p[3].y));
      }
    }
    // the two halves' partial sums meet in shared memory (every epilogue
    // thread reaches this barrier, also after a timeout)
    if (half == 1) s_part[m] = partial;
    asm volatile("bar.sync 1, %0;\n" ::"n"(kEpiWarps * 32) : "memory");
    if (half == 0 && ok && !s_abort) {
      const int gm = row0 + m;
      if (gm < a.batch) a.out[gm] = a.p32[a.b_off[nhid]] + (partial + s_part[m]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (s_abort && threadIdx.x == 0 && a.status != nullptr) atomicExch(a.status, FLPR_ERR_TIMEOUT);
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

constexpr size_t kTcSmem = 1024 /* alignment */ + (size_t)kMaxInChunks * kAChunk +
                           (size_t)kStages * kBChunk +
                           (2 * kStages + kMaxInChunks + 1 + kHidChunks) * sizeof(uint64_t) +
                           4 * sizeof(uint32_t) + sizeof(float) * (size_t)(kMaxLayersTc * kHid + kTM);
// the float4 reads of the bias cache need it on a 16-byte boundary
static_assert(((size_t)kMaxInChunks * kAChunk + (size_t)kStages * kBChunk +
               (2 * kStages + kMaxInChunks + 1 + kHidChunks) * sizeof(uint64_t) +
               4 * sizeof(uint32_t)) % 16 == 0, "bias cache alignment");

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_fn(EncodeTiledFn* out) {
  static EncodeTiledFn fn = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (fn == nullptr) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    FLPR_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    FLPR_CHECK_ARG(q == cudaDriverEntryPointSuccess && p != nullptr,
                   "mlp_infer: driver entry point cuTensorMapEncodeTiled missing");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  *out = fn;
  return FLPR_OK;
}

// K-major BF16 matrix of `rows` rows and K columns (row stride K elements)
// read in boxes of 64 columns x box_rows rows with the 128-byte swizzle;
// entries outside the matrix read as zero
static int encode_bf16_2d(EncodeTiledFn fn, CUtensorMap* tm, const void* base, int K, int rows,
                          int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kKC, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  FLPR_CHECK_ARG(r == CUDA_SUCCESS, "mlp_infer: cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FLPR_OK;
}

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
    // tensor maps start on 16-byte boundaries
    FLPR_CHECK_ARG(((uintptr_t)d_params16 + 2 * (uintptr_t)a.w_off[l]) % 16 == 0,
                   "mlp_infer: weights of layer %d not 16-byte aligned", l);
  }
  FLPR_CHECK_ARG((uintptr_t)d_x16 % 16 == 0, "mlp_infer: inputs not 16-byte aligned");
  a.total_chunks = 0;
  for (int l = 0; l < nlayers - 1; ++l) {
    a.nchunks[l] = (h_dims[l] + kKC - 1) / kKC;
    a.total_chunks += a.nchunks[l];
  }
  EncodeTiledFn fn = nullptr;
  FLPR_TRY(encode_fn(&fn));
  const __nv_bfloat16* p16 = static_cast<const __nv_bfloat16*>(d_params16);
  for (int l = 0; l < nlayers - 1; ++l)
    FLPR_TRY(encode_bf16_2d(fn, &a.tm_w[l], p16 + a.w_off[l], h_dims[l], kHid, kHid));
  // a batch smaller than the tile copies only its own rows (rounded up to
  // 8): the tile's other rows hold stale values, whose products land in
  // accumulator rows that no output reads (every row of D depends on its
  // own row of A alone)
  a.in_box_rows = batch >= kTM ? kTM : ((batch + 7) / 8) * 8;
  FLPR_TRY(encode_bf16_2d(fn, &a.tm_x, d_x16, h_dims[0], batch, a.in_box_rows));
  a.batch = batch;
  a.p16 = p16;
  a.p32 = d_params32;
  a.out = d_out;
  a.status = d_status;
  FLPR_CUDA(raise_dyn_smem(mlp_infer_tc_kernel, kTcSmem));
  const int grid = (batch + kTM - 1) / kTM;
  mlp_infer_tc_kernel<<<grid, kThreads, kTcSmem, as_stream(stream)>>>(a);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
