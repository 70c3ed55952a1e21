// cuFFT plan cache: plans are created without work areas (the caller's
// workspace is attached at execution), keyed by shape, type and batch.
#pragma once

#include "common.cuh"

namespace flpr {

struct PlanKey {
  int rank;
  int n[3];
  int type;   // cufftType
  int batch;
  int idist;
  int odist;
  int stride;   // element stride of input and output (0 or 1: contiguous)
  int inverse;  // C2C / Z2Z direction
  bool operator<(const PlanKey& o) const {
    return std::tie(rank, n[0], n[1], n[2], type, batch, idist, odist, stride, inverse) <
           std::tie(o.rank, o.n[0], o.n[1], o.n[2], o.type, o.batch, o.idist, o.odist, o.stride,
                    o.inverse);
  }
};

struct Plan {
  cufftHandle plan = 0;
  size_t work = 0;
};

struct PlanCache {
  std::mutex mu;
  std::map<PlanKey, Plan> plans;
  ~PlanCache();
  int get(const PlanKey& key, Plan** out);
  int exec(const PlanKey& key, void* in, void* out, void* work, size_t work_bytes,
           cudaStream_t stream);
  int work_size(const PlanKey& key, size_t* out);
};

PlanCache& plans_of(flpr_handle_t h);

// Real/complex transform over all axes of an L^d grid, batched.
inline PlanKey grid_plan(int d, const int* L, int type, int batch) {
  PlanKey k{};
  k.rank = d;
  for (int i = 0; i < 3; ++i) k.n[i] = i < d ? L[i] : 0;
  int64_t real = 1, cplx = 1;
  for (int i = 0; i < d; ++i) {
    real *= L[i];
    cplx *= (i == d - 1) ? (L[i] / 2 + 1) : L[i];
  }
  k.type = type;
  k.batch = batch;
  bool fwd = (type == CUFFT_R2C || type == CUFFT_D2Z);
  k.idist = (int)(fwd ? real : cplx);
  k.odist = (int)(fwd ? cplx : real);
  return k;
}

}  // namespace flpr
