// Point statistics and small elementwise helpers.
#include "common.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

namespace flpr {

struct Moments {
  double n, mean, m2, lo, hi;
};

__device__ __forceinline__ Moments merge(const Moments& a, const Moments& b) {
  if (a.n == 0) return b;
  if (b.n == 0) return a;
  Moments r;
  r.n = a.n + b.n;
  double delta = b.mean - a.mean;
  r.mean = a.mean + delta * (b.n / r.n);
  r.m2 = a.m2 + b.m2 + delta * delta * (a.n * b.n / r.n);
  r.lo = fmin(a.lo, b.lo);
  r.hi = fmax(a.hi, b.hi);
  return r;
}

constexpr int kStatThreads = 256;

// One block-partial per (block, axis): Welford per thread, Chan merge.
__global__ void point_stats_partial(int d, int64_t n, const double* __restrict__ x,
                                    Moments* __restrict__ part) {
  __shared__ Moments sh[kStatThreads];
  for (int ax = 0; ax < d; ++ax) {
    Moments m{0.0, 0.0, 0.0, INFINITY, -INFINITY};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
      double v = x[i * d + ax];
      m.n += 1.0;
      double delta = v - m.mean;
      m.mean += delta / m.n;
      m.m2 += delta * (v - m.mean);
      m.lo = fmin(m.lo, v);
      m.hi = fmax(m.hi, v);
    }
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sh[threadIdx.x] = merge(sh[threadIdx.x], sh[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x * d + ax] = sh[0];
    __syncthreads();
  }
}

__global__ void point_stats_final(int d, int nblocks, const Moments* __restrict__ part,
                                  double* __restrict__ out) {
  __shared__ Moments sh[kStatThreads];
  for (int ax = 0; ax < d; ++ax) {
    Moments m{0.0, 0.0, 0.0, INFINITY, -INFINITY};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) m = merge(m, part[b * d + ax]);
    sh[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sh[threadIdx.x] = merge(sh[threadIdx.x], sh[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      out[ax] = sh[0].lo;
      out[d + ax] = sh[0].hi;
      out[2 * d + ax] = sh[0].mean;
      out[3 * d + ax] = sh[0].m2;
    }
    __syncthreads();
  }
}

static int stat_blocks(int64_t n) {
  int64_t b = (n + kStatThreads - 1) / kStatThreads;
  int64_t cap = 4 * (int64_t)sm_count();
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

__global__ void log_shift_kernel(int64_t n, const double* __restrict__ in, double shift,
                                 double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = log(in[i] + shift);
}

__global__ void exp_weighted_sum_kernel(int64_t n, const double* __restrict__ yraw,
                                        const double* __restrict__ yhat, double* __restrict__ acc) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += yraw[i] * exp(-yhat[i]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(acc, sh[0]);
}

// ---- allocation-free variant of the point statistics ----------------------
// Scratch of flpr_point_stats_noalloc: one Moments record per (block, axis),
// kNoAllocMaxBlocks x kNoAllocMaxDims records (320 KiB).  It lives in the
// library's own device data, so every GPU that loads the library holds it
// until the process exits.
constexpr int kNoAllocMaxBlocks = 1024;
constexpr int kNoAllocMaxDims = 8;
static __device__ __align__(256) Moments g_noalloc_partials[kNoAllocMaxBlocks * kNoAllocMaxDims];

// Device address of g_noalloc_partials, looked up once per device context.
// Host code must not pass the symbol itself to a kernel: on the host it is
// only a stand-in.  The cache is keyed by the unique id of the current
// context (cuCtxGetId), so a context created after a device reset, or a
// caller's own driver-API context, looks the address up again.
constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
struct NoAllocSlot {
  unsigned long long ctx_id;
  Moments* addr;
};
static NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices] = {};

// Unique id of the current context (0 when none is current yet).  Resolved
// through the runtime's driver entry points, so the library does not link
// the driver library itself.
static int current_context_id(unsigned long long* id) {
  static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  if (get_current == nullptr || get_id == nullptr) {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    FLPR_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault,
                                      &q1));
    FLPR_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2));
    FLPR_CHECK_ARG(q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess,
                   "point_stats_noalloc: driver entry points cuCtxGetCurrent/cuCtxGetId missing");
  }
  CUcontext ctx = nullptr;
  FLPR_CHECK_ARG(get_current(&ctx) == CUDA_SUCCESS, "point_stats_noalloc: cuCtxGetCurrent failed");
  *id = 0;
  if (ctx != nullptr)
    FLPR_CHECK_ARG(get_id(ctx, id) == CUDA_SUCCESS, "point_stats_noalloc: cuCtxGetId failed");
  return FLPR_OK;
}

static int noalloc_scratch(Moments** out) {
  int dev = 0;
  FLPR_CUDA(cudaGetDevice(&dev));
  FLPR_CHECK_ARG(dev >= 0 && dev < kNoAllocMaxDevices, "point_stats_noalloc: device %d", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  unsigned long long id = 0;
  FLPR_TRY(current_context_id(&id));
  NoAllocSlot& slot = g_noalloc_slot[dev];
  if (id == 0 || slot.addr == nullptr || slot.ctx_id != id) {
    // the lookup makes the device's primary context current when none is
    void* p = nullptr;
    FLPR_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partials));
    FLPR_TRY(current_context_id(&id));
    slot.addr = static_cast<Moments*>(p);
    slot.ctx_id = id;
  }
  *out = slot.addr;
  return FLPR_OK;
}

}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_point_stats_noalloc(int d, int64_t n, const double* d_x, double* d_stats, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= kNoAllocMaxDims,
                 "point_stats_noalloc: d=%d exceeds the static scratch (max %d axes)", d,
                 kNoAllocMaxDims);
  FLPR_CHECK_ARG(n >= 1, "point_stats_noalloc: n=%lld", (long long)n);
  int nb = stat_blocks(n);
  if (nb > kNoAllocMaxBlocks) nb = kNoAllocMaxBlocks;  // grid-stride loop covers any n
  Moments* part = nullptr;
  FLPR_TRY(noalloc_scratch(&part));
  // every block writes its record for every axis before point_stats_final
  // reads it, so nothing in the scratch has to start at zero
  point_stats_partial<<<nb, kStatThreads, 0, as_stream(stream)>>>(d, n, d_x, part);
  FLPR_LAUNCH_CHECK();
  point_stats_final<<<1, kStatThreads, 0, as_stream(stream)>>>(d, nb, part, d_stats);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

size_t flpr_point_stats_ws(int d, int64_t n) {
  return align_up(sizeof(Moments) * (size_t)stat_blocks(n) * (size_t)(d > 0 ? d : 1));
}

int flpr_point_stats(int d, int64_t n, const double* d_x, double* d_stats, void* d_ws,
                     size_t ws_bytes, void* stream) {
  FLPR_CHECK_ARG(d >= 1 && d <= 16, "point_stats: bad d=%d", d);
  FLPR_CHECK_ARG(n >= 1, "point_stats: n=%lld", (long long)n);
  if (ws_bytes < flpr_point_stats_ws(d, n)) {
    set_error("point_stats: workspace too small");
    return FLPR_ERR_WORKSPACE;
  }
  int nb = stat_blocks(n);
  Moments* part = static_cast<Moments*>(d_ws);
  point_stats_partial<<<nb, kStatThreads, 0, as_stream(stream)>>>(d, n, d_x, part);
  FLPR_LAUNCH_CHECK();
  point_stats_final<<<1, kStatThreads, 0, as_stream(stream)>>>(d, nb, part, d_stats);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_log_shift(int64_t n, const double* d_in, double shift, double* d_out, void* stream) {
  FLPR_CHECK_ARG(n >= 1, "log_shift: n=%lld", (long long)n);
  int nb = (int)((n + 255) / 256);
  if (nb > 8 * sm_count()) nb = 8 * sm_count();
  log_shift_kernel<<<nb, 256, 0, as_stream(stream)>>>(n, d_in, shift, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

int flpr_exp_weighted_sum(int64_t n, const double* d_yraw, const double* d_yhat, double* d_acc,
                          void* stream) {
  FLPR_CHECK_ARG(n >= 1, "exp_weighted_sum: n=%lld", (long long)n);
  FLPR_CUDA(cudaMemsetAsync(d_acc, 0, sizeof(double), as_stream(stream)));
  int nb = (int)((n + 255) / 256);
  if (nb > 4 * sm_count()) nb = 4 * sm_count();
  exp_weighted_sum_kernel<<<nb, 256, 0, as_stream(stream)>>>(n, d_yraw, d_yhat, d_acc);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
