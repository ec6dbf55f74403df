// Library-wide C-ABI entry points: version, last error, launch counter.
#include "pe_internal.h"

namespace pe {

std::string &last_error() {
  thread_local std::string message;
  return message;
}

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  last_error() = buf;
  return code;
}

int cuda_fail(cudaError_t err, const char *what) {
  const int code =
      err == cudaErrorMemoryAllocation ? PE_ENOMEM : PE_ECUDA;
  return fail(code, "%s: %s", what, cudaGetErrorString(err));
}

static std::atomic<int64_t> g_launches{0};

void count_launches(int64_t n) { g_launches.fetch_add(n); }

}  // namespace pe

extern "C" {

int pe_version(void) { return PE_ABI_VERSION; }

const char *pe_last_error(void) { return pe::last_error().c_str(); }

int64_t pe_launch_count(void) { return pe::g_launches.load(); }

}  // extern "C"

namespace pe {

LaunchTimer::~LaunchTimer() {
  for (auto &pr : pending_) {
    cudaEventDestroy(pr.start);
    cudaEventDestroy(pr.stop);
  }
  for (auto e : spare_) cudaEventDestroy(e);
}

cudaEvent_t LaunchTimer::take() {
  if (!spare_.empty()) {
    cudaEvent_t e = spare_.back();
    spare_.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

cudaEvent_t LaunchTimer::begin(cudaStream_t stream) {
  if (!enabled_) return nullptr;
  cudaEvent_t e = take();
  if (e && cudaEventRecord(e, stream) != cudaSuccess) {
    spare_.push_back(e);
    return nullptr;
  }
  return e;
}

int LaunchTimer::end(cudaStream_t stream, cudaEvent_t start, int slot) {
  if (!enabled_ || !start) return PE_OK;
  cudaEvent_t stop = take();
  if (!stop) return fail(PE_ECUDA, "profiling: cannot create an event");
  PE_CUDA_TRY(cudaEventRecord(stop, stream));
  pending_.push_back({start, stop, slot});
  if (pending_.size() > kSoftCap) return harvest(pending_.size() > kHardCap);
  return PE_OK;
}

int LaunchTimer::harvest(bool wait_all) {
  while (!pending_.empty()) {
    Pair pr = pending_.front();
    if (wait_all) {
      PE_CUDA_TRY(cudaEventSynchronize(pr.stop));
    } else {
      const cudaError_t q = cudaEventQuery(pr.stop);
      if (q == cudaErrorNotReady) {
        (void)cudaGetLastError();  // not an error: clear it
        break;
      }
      if (q != cudaSuccess) return cuda_fail(q, "profiling event");
    }
    float ms = 0;
    PE_CUDA_TRY(cudaEventElapsedTime(&ms, pr.start, pr.stop));
    ms_[pr.slot] += ms;
    n_[pr.slot] += 1;
    spare_.push_back(pr.start);
    spare_.push_back(pr.stop);
    pending_.pop_front();
  }
  return PE_OK;
}

int LaunchTimer::reset(bool enable) {
  const int rc = harvest(true);
  if (rc) return rc;
  enabled_ = enable;
  for (int s = 0; s < kSlots; s++) {
    ms_[s] = 0;
    n_[s] = 0;
  }
  return PE_OK;
}

}  // namespace pe
