// Shared helpers for the fastlpr_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/fastlpr_b200.h"

namespace flpr {

// Per-thread message for flpr_last_error().
void set_error(const char* fmt, ...);

// Number of kernels this library has launched (flpr_launch_count()).
void count_launch();
// process-wide tuning parameters (flpr_set_tuning)
int tuning(int param);

#define FLPR_CHECK_ARG(cond, ...)            \
  do {                                       \
    if (!(cond)) {                           \
      ::flpr::set_error(__VA_ARGS__);        \
      return FLPR_ERR_ARG;                   \
    }                                        \
  } while (0)

#define FLPR_CUDA(call)                                                        \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ::flpr::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                        cudaGetErrorString(e_));                               \
      return FLPR_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

#define FLPR_LAUNCH_CHECK()                                                    \
  do {                                                                         \
    ::flpr::count_launch();                                                    \
    cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess) {                                                   \
      ::flpr::set_error("%s:%d launch: %s", __FILE__, __LINE__,                \
                        cudaGetErrorString(e_));                               \
      return FLPR_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

#define FLPR_CUFFT(call)                                                       \
  do {                                                                         \
    cufftResult r_ = (call);                                                   \
    if (r_ != CUFFT_SUCCESS) {                                                 \
      ::flpr::set_error("%s:%d %s: cufft error %d", __FILE__, __LINE__, #call, \
                        (int)r_);                                              \
      return FLPR_ERR_CUFFT;                                                   \
    }                                                                          \
  } while (0)

#define FLPR_TRY(call)                 \
  do {                                 \
    int s_ = (call);                   \
    if (s_ != FLPR_OK) return s_;      \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline size_t align_up(size_t v, size_t a = 256) { return (v + a - 1) / a * a; }

// Bump allocator over a caller-provided workspace.
struct Arena {
  char* base;
  size_t size;
  size_t used = 0;
  Arena(void* b, size_t s) : base(static_cast<char*>(b)), size(s) {}
  template <typename T>
  T* take(size_t count) {
    size_t off = align_up(used);
    used = off + align_up(count * sizeof(T));
    if (used > size) return nullptr;
    return reinterpret_cast<T*>(base + off);
  }
};

// Size-only counterpart of Arena for *_ws queries.
struct ArenaSize {
  size_t used = 0;
  template <typename T>
  T* take(size_t count) {
    used = align_up(used) + align_up(count * sizeof(T));
    return nullptr;
  }
};

inline int sm_count() {
  static int cached = -1;
  if (cached < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached = v;
  }
  return cached;
}

// Raise the dynamic shared-memory limit of `kernel` on the current device
// to at least `bytes`.  The limit never goes down: a launch is checked
// against the limit in force when it starts, so a launch captured in a CUDA
// graph (or a profiler's replay of it) with a larger size stays valid after
// a later launch of the same kernel asked for less.
template <typename K>
inline cudaError_t raise_dyn_smem(K kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limit_of;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& lim = limit_of[std::make_pair(dev, reinterpret_cast<const void*>(kernel))];
  if (bytes <= lim) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) lim = bytes;
  return e;
}

// Shared-memory carveout of `kernel` sized for as many CTAs per SM as its
// registers and `dyn_smem` allow at the largest carveout; the rest of the
// unified L1/shared array stays L1.  Both attributes are set on every call
// (another size may have been set since); the occupancy query runs once per
// (device, kernel, size, threads).
template <typename K>
inline cudaError_t fit_carveout(K kernel, int threads, size_t dyn_smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, size_t, int>, int> pct_of;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = raise_dyn_smem(kernel, dyn_smem)) != cudaSuccess) return e;
  const auto key = std::make_tuple(dev, reinterpret_cast<const void*>(kernel), dyn_smem, threads);
  int pct = -1;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = pct_of.find(key);
    if (it != pct_of.end()) pct = it->second;
  }
  if (pct < 0) {
    if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
      return e;
    int blocks = 0, per_sm = 0, reserved = 0;
    cudaFuncAttributes fa;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, dyn_smem)) !=
            cudaSuccess ||
        (e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) !=
            cudaSuccess ||
        (e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) !=
            cudaSuccess ||
        (e = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess)
      return e;
    pct = 100;
    if (blocks > 0 && per_sm > 0) {
      const size_t need = (size_t)blocks * (dyn_smem + fa.sharedSizeBytes + (size_t)reserved);
      pct = (int)((need * 100 + (size_t)per_sm - 1) / (size_t)per_sm);
      pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
    }
    std::lock_guard<std::mutex> lk(mu);
    pct_of[key] = pct;
  }
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

inline int64_t prod(const int* v, int d) {
  int64_t p = 1;
  for (int i = 0; i < d; ++i) p *= v[i];
  return p;
}

// Round-to-nearest FP64 arithmetic without contraction into FMA; the knot
// mapping must reproduce the reference's elementwise numpy operations.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// numpy.mod for float64 (floor-style remainder).
__device__ __forceinline__ double np_mod(double a, double b) {
  double r = fmod(a, b);
  if (r != 0.0) {
    if ((b < 0.0) != (r < 0.0)) r = dadd(r, b);
  } else {
    r = copysign(0.0, b);
  }
  return r;
}

// Per-axis knot map constants, in the order of flpr_spread's h_kmap.
struct KnotAxis {
  double mean, std, center, xs_min, xs_scale, ks, r0, shift, hx;
};

// Knot coordinate of raw coordinate x on one axis (see the header).
__device__ __forceinline__ double knot_of(double x, const KnotAxis& a) {
  double xs = dsub(ddiv(dsub(x, a.mean), a.std), a.center);
  double xn = dadd(dmul(ddiv(dsub(xs, a.xs_min), a.xs_scale), a.ks), a.r0);
  xn = dadd(xn, 0.5);
  xn = np_mod(xn, 1.0);
  double k = dsub(xn, 0.5);
  k = dadd(k, a.shift);
  k = dmul(k, 6.283185307179586);  // 2*pi as the float64 numpy computes it
  return np_mod(k, 6.283185307179586);
}

}  // namespace flpr
