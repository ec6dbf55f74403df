// Internal host helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

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

}  // namespace pe

#define PE_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t pe_err_ = (expr);                           \
    if (pe_err_ != cudaSuccess) return pe::cuda_fail(pe_err_, #expr); \
  } while (0)
