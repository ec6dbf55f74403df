// Internal host helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <deque>
#include <string>
#include <vector>

#include "pe_b200.h"

namespace pe {

// Message of the last failure on this thread, returned by pe_last_error().
std::string &last_error();

// Record a failure message and return `code`.
int fail(int code, const char *fmt, ...);

// Map a CUDA error to PE_ENOMEM / PE_ECUDA with a message naming `what`.
int cuda_fail(cudaError_t err, const char *what);

// Count of kernels this library has launched (pe_launch_count()).
void count_launches(int64_t n);

// Per-launch device time from CUDA event pairs recorded on the launching
// stream, summed per slot (e.g. RK2 stage 1 / stage 2).  Finished pairs are
// harvested without blocking once many are outstanding, so profiling adds
// no host synchronisation to a long run unless the device falls more than
// kHardCap launches behind.
class LaunchTimer {
 public:
  static constexpr size_t kSoftCap = 1024, kHardCap = 65536;
  static constexpr int kSlots = 2;

  ~LaunchTimer();
  // Event to record before the launch (nullptr when disabled).
  cudaEvent_t begin(cudaStream_t stream);
  // Record the end event after the launch and file the pair under `slot`.
  int end(cudaStream_t stream, cudaEvent_t start, int slot);
  // Sum finished pairs; wait_all waits for every outstanding pair.
  int harvest(bool wait_all);
  // Wait for outstanding pairs, zero the sums and switch on or off.
  int reset(bool enable);
  bool enabled() const { return enabled_; }
  double ms(int slot) const { return ms_[slot]; }
  int64_t launches(int slot) const { return n_[slot]; }

 private:
  struct Pair {
    cudaEvent_t start, stop;
    int slot;
  };
  cudaEvent_t take();
  bool enabled_ = false;
  double ms_[kSlots] = {0, 0};
  int64_t n_[kSlots] = {0, 0};
  std::deque<Pair> pending_;
  std::vector<cudaEvent_t> spare_;
};

}  // namespace pe

#define PE_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t pe_err_ = (expr);                           \
    if (pe_err_ != cudaSuccess) return pe::cuda_fail(pe_err_, #expr); \
  } while (0)
