// Legacy six-dimensional square game (src/pursuit_evasion/dp/native_square.cpp):
// shared declarations of the exact stage kernel and the C-ABI handle.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pe {

struct Square6Grid {
  int n, nh, order;
  int64_t cells;
  int64_t stride[6];  // [xP, yP, thP, xE, yE, thE], thE fastest
  float dx, dh;       // native_square.cpp:87
  // 1/dx, 1/(dx*dx), 1/dh, 1/(dh*dh) rounded to nearest (squares rounded in
  // float): the exact stage's divisions go through them (div_rn.cuh)
  float rdx, rdx2, rdh, rdh2;
  float vp, ve, wp, we, arena;
};

struct Square6Stats {
  unsigned long long residual;  // bits of a non-negative double: max |change|
  unsigned int nonfinite;
  unsigned int pad;
};

struct Square6Stage {
  const float *src;
  float *dst;
  const float *base;  // RK2 average partner (nullptr on the first stage)
  float *arrival;
  const float *x, *cs, *sn;  // float axes (native_square.cpp:98-104)
  float dt;
  double tau;
  Square6Stats *stats;
};

// One stage in the reference's float32 operation order (bit for bit).
cudaError_t square6_stage(const Square6Grid &g, const Square6Stage &s, cudaStream_t stream);

// field = block[(xP, yP, xE, yE)] repeated over both headings; arrival 0
// where <= 0, else NaN.
cudaError_t square6_init(const Square6Grid &g, const float *block, float *field,
                         float *arrival, cudaStream_t stream);

}  // namespace pe
