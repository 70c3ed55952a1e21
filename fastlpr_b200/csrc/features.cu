// Binned moment sums of a data set, the input summary of the bandwidth
// proposal network: on a grid of 4096 cells spanning [min, max] of every
// axis (4096 bins in 1-D, 64 x 64 in 2-D), the count, sum y and sum y^2 of
// the points in each cell.
#include "common.cuh"

namespace flpr {
namespace {

constexpr int kFeatCells = 4096;
__host__ __device__ constexpr int feat_bins(int d) { return d == 1 ? 4096 : 64; }

// grid-stride over the points; per-block float histogram in shared memory,
// flushed to the FP64 output with one atomic per non-zero cell
__global__ void bin_moments_kernel(int d, int64_t n, const double* __restrict__ x,
                                   const double* __restrict__ y, const double* __restrict__ stats,
                                   double* __restrict__ out) {
  extern __shared__ float hist[];  // 3 x cells
  const int cells = kFeatCells, bins = feat_bins(d);
  for (int i = threadIdx.x; i < 3 * cells; i += blockDim.x) hist[i] = 0.0f;
  __syncthreads();
  double lo[2], scale[2];
  for (int a = 0; a < d; ++a) {
    lo[a] = stats[a];
    const double span = stats[d + a] - stats[a];
    scale[a] = span > 0.0 ? (double)bins / span : 0.0;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int cell = 0;
    for (int a = 0; a < d; ++a) {
      int b = (int)floor((x[i * d + a] - lo[a]) * scale[a]);
      b = b < 0 ? 0 : (b >= bins ? bins - 1 : b);
      cell = cell * bins + b;
    }
    const float v = (float)y[i];
    atomicAdd(&hist[cell], 1.0f);
    atomicAdd(&hist[cells + cell], v);
    atomicAdd(&hist[2 * cells + cell], v * v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * cells; i += blockDim.x)
    if (hist[i] != 0.0f) atomicAdd(&out[i], (double)hist[i]);
}

}  // namespace
}  // namespace flpr

using namespace flpr;

extern "C" {

int flpr_bin_moments(int d, int64_t n, const double* d_x, const double* d_y, const double* d_stats,
                     double* d_out, void* stream) {
  FLPR_CHECK_ARG(d == 1 || d == 2, "bin_moments: d=%d (1 or 2)", d);
  FLPR_CHECK_ARG(n >= 1, "bin_moments: n=%lld", (long long)n);
  const int cells = kFeatCells;
  cudaStream_t s = as_stream(stream);
  FLPR_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * 3 * cells, s));
  const size_t smem = sizeof(float) * 3 * cells;
  int nb = (int)((n + 1023) / 1024);
  if (nb > 2 * sm_count()) nb = 2 * sm_count();
  if (nb < 1) nb = 1;
  bin_moments_kernel<<<nb, 256, smem, s>>>(d, n, d_x, d_y, d_stats, d_out);
  FLPR_LAUNCH_CHECK();
  return FLPR_OK;
}

}  // extern "C"
