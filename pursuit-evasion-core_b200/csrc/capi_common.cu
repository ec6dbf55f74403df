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
