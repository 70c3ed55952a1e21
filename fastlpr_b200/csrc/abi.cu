// Handle, error reporting and cuFFT plan cache.
#include <stdarg.h>

#include <atomic>

#include "common.cuh"
#include "plans.cuh"

namespace flpr {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// defaults and ranges of the FLPR_TUNE_* parameters
static std::atomic<int> g_tune[FLPR_TUNE_COUNT] = {{4096}, {768}};
static const int kTuneMin[FLPR_TUNE_COUNT] = {256, 8};
static const int kTuneMax[FLPR_TUNE_COUNT] = {65536, 16384};

int tuning(int param) { return g_tune[param].load(std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

PlanCache::~PlanCache() {
  for (auto& kv : plans) cufftDestroy(kv.second.plan);
}

int PlanCache::get(const PlanKey& key, Plan** out) {
  std::lock_guard<std::mutex> lock(mu);
  auto it = plans.find(key);
  if (it != plans.end()) {
    *out = &it->second;
    return FLPR_OK;
  }
  Plan p;
  FLPR_CUFFT(cufftCreate(&p.plan));
  FLPR_CUFFT(cufftSetAutoAllocation(p.plan, 0));
  int rank = key.rank;
  int n[3] = {key.n[0], key.n[1], key.n[2]};
  size_t ws = 0;
  const int stride = key.stride > 1 ? key.stride : 1;
  int emb[3] = {n[0], n[1], n[2]};
  cufftResult r = cufftMakePlanMany(p.plan, rank, n, stride > 1 ? emb : nullptr, stride, key.idist,
                                    stride > 1 ? emb : nullptr, stride, key.odist,
                                    static_cast<cufftType>(key.type), key.batch, &ws);
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(p.plan);
    set_error("cufftMakePlanMany(rank=%d n=%d,%d,%d type=%d batch=%d) failed: %d", rank, n[0],
              n[1], n[2], key.type, key.batch, (int)r);
    return FLPR_ERR_CUFFT;
  }
  p.work = ws;
  auto res = plans.emplace(key, p);
  *out = &res.first->second;
  return FLPR_OK;
}

int PlanCache::exec(const PlanKey& key, void* in, void* out, void* work, size_t work_bytes,
                    cudaStream_t stream) {
  Plan* p = nullptr;
  FLPR_TRY(get(key, &p));
  if (work_bytes < p->work) {
    set_error("cuFFT work area %zu < required %zu", work_bytes, p->work);
    return FLPR_ERR_WORKSPACE;
  }
  FLPR_CUFFT(cufftSetStream(p->plan, stream));
  FLPR_CUFFT(cufftSetWorkArea(p->plan, work));
  switch (key.type) {
    case CUFFT_R2C:
      FLPR_CUFFT(cufftExecR2C(p->plan, (cufftReal*)in, (cufftComplex*)out));
      break;
    case CUFFT_C2R:
      FLPR_CUFFT(cufftExecC2R(p->plan, (cufftComplex*)in, (cufftReal*)out));
      break;
    case CUFFT_D2Z:
      FLPR_CUFFT(cufftExecD2Z(p->plan, (cufftDoubleReal*)in, (cufftDoubleComplex*)out));
      break;
    case CUFFT_Z2D:
      FLPR_CUFFT(cufftExecZ2D(p->plan, (cufftDoubleComplex*)in, (cufftDoubleReal*)out));
      break;
    case CUFFT_Z2Z:
      FLPR_CUFFT(cufftExecZ2Z(p->plan, (cufftDoubleComplex*)in, (cufftDoubleComplex*)out,
                              key.inverse ? CUFFT_INVERSE : CUFFT_FORWARD));
      break;
    case CUFFT_C2C:
      FLPR_CUFFT(cufftExecC2C(p->plan, (cufftComplex*)in, (cufftComplex*)out,
                              key.inverse ? CUFFT_INVERSE : CUFFT_FORWARD));
      break;
    default:
      set_error("unsupported FFT type %d", key.type);
      return FLPR_ERR_ARG;
  }
  return FLPR_OK;
}

int PlanCache::work_size(const PlanKey& key, size_t* out) {
  Plan* p = nullptr;
  FLPR_TRY(get(key, &p));
  *out = p->work;
  return FLPR_OK;
}

}  // namespace flpr

struct flpr_handle_s {
  int device;
  flpr::PlanCache plans;
};

namespace flpr {
PlanCache& plans_of(flpr_handle_t h) { return h->plans; }
}  // namespace flpr

extern "C" {

const char* flpr_last_error(void) { return flpr::g_err; }

int flpr_version(void) { return 100; }

int64_t flpr_launch_count(void) { return (int64_t)flpr::g_launches.load(); }

int flpr_set_tuning(int param, int value) {
  FLPR_CHECK_ARG(param >= 0 && param < FLPR_TUNE_COUNT, "set_tuning: param=%d", param);
  FLPR_CHECK_ARG(value >= flpr::kTuneMin[param] && value <= flpr::kTuneMax[param],
                 "set_tuning: value %d of param %d outside [%d, %d]", value, param,
                 flpr::kTuneMin[param], flpr::kTuneMax[param]);
  flpr::g_tune[param].store(value, std::memory_order_relaxed);
  return FLPR_OK;
}

int flpr_get_tuning(int param) {
  if (param < 0 || param >= FLPR_TUNE_COUNT) return -1;
  return flpr::tuning(param);
}

int flpr_create(flpr_handle_t* out, int device) {
  FLPR_CHECK_ARG(out != nullptr, "flpr_create: null output pointer");
  FLPR_CUDA(cudaSetDevice(device));
  flpr_handle_s* h = new flpr_handle_s();
  h->device = device;
  *out = h;
  return FLPR_OK;
}

int flpr_destroy(flpr_handle_t handle) {
  delete handle;
  return FLPR_OK;
}

}  // extern "C"
