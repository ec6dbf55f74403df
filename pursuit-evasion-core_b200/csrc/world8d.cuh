// Dense 8D ENO/Lax-Friedrichs capture step: shared declarations.
//
// Storage order [xP, yP, thP, vP, xE, yE, thE, vE] with vE fastest, float32
// (the layout of native_world.cpp:122-136 and of world tables).  One launch
// = one stage of the RK1/RK2 update of native_world.cpp:261-314.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pe {

struct World8Grid {
  int n, nh, np, ne, order;
  int linear_speed;  // inward one-sided slopes at the speed bounds
  int avoid_mode;    // 0: none; 1: square arena max(|xP|,|yP|) - arena + 1e-6;
                     // 2: obstacle clearance -p_clear[xP, yP, thP] + 1e-6
  int64_t cells;
  int64_t stride[8];
  int shape[8];
  float spacing[8];
  float inv_spacing[8];     // 1 / spacing rounded to nearest
  float inv_spacing_sq[8];  // 1 / (spacing * spacing) rounded to nearest (the
                            // square rounded in float, as the stage forms it)
  float extent, arena, ap, ae, kp, ke;
};

struct World8Stats {
  unsigned long long residual;  // bits of a non-negative double
  unsigned int nonfinite;
  unsigned int pad;
};

struct World8Stage {
  const float *src;
  float *dst;
  const float *base;  // RK2 average partner (nullptr on the first stage)
  float *arrival;
  const float *x, *cs, *sn, *pv, *ev;  // float axes (native_world.cpp:138-150)
  float dt;
  double tau;
  World8Stats *stats;
  const float *p_clear;  // avoid_mode 2: pursuer clearance [xP][yP][thP]
};

// One stage in float32 arithmetic evaluated in the reference's order; the
// translation unit is built without multiply-add contraction, so results
// equal native_world.cpp's bit for bit.
cudaError_t world8_stage(const World8Grid &g, const World8Stage &s,
                         cudaStream_t stream);

// The same stage with reciprocal spacings and multiply-add contraction:
// equal to the exact stage up to float rounding (and the ENO2 selections
// rounding can flip).
cudaError_t world8_stage_fast(const World8Grid &g, const World8Stage &s,
                              cudaStream_t stream);

// Capture field of the 8D contact game: the oriented-rectangle separation of
// the two footprints at every grid pose, in double, stored as float; arrival
// = 0 where <= 0.  cs/sn: double cos/sin of the heading axis; cdiff/sdiff:
// cos/sin of (thE - thP) for every heading pair, [thE * nh + thP].
cudaError_t world8_init_contact(const World8Grid &g, const double *cs,
                                const double *sn, const double *cdiff,
                                const double *sdiff, double p_len, double p_wid,
                                double e_len, double e_wid, float *field,
                                float *arrival, cudaStream_t stream);

// The reference's square-arena surfaces (native_world.cpp:155-176):
// max(min(capture, E fault), P avoid).
cudaError_t world8_init_square(const World8Grid &g, const float *x,
                               float radius, float *field, float *arrival,
                               cudaStream_t stream);

// The obstacle map game's surfaces (gpu_map_game.py:45-50): centre-distance
// capture limited by the evader's clearance, floored by the pursuer's
// clearance: max(min(hypot(dxP - dxE) - r, e_clear), -p_clear + 1e-6), the
// clearances per (x, y, heading) pose of each car.
cudaError_t world8_init_map(const World8Grid &g, float radius, const float *p_clear,
                            const float *e_clear, float *field, float *arrival,
                            cudaStream_t stream);

// arrival = start where field <= 0, NaN elsewhere (after a host upload).
cudaError_t world8_init_arrival(const World8Grid &g, const float *field,
                                float *arrival, float start,
                                cudaStream_t stream);

}  // namespace pe
