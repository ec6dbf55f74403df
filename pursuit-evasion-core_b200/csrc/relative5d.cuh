// Relative 5D ENO/Lax-Friedrichs capture-tube kernels: shared declarations.
//
// Storage order [vP, vE, psi, y, x], x fastest (the reference's fields.f32
// frame layout, free_dp.py:45-54).  One launch = one stage of the RK1/RK2
// update of native_relative.cpp:124-172 over every cell.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pe {

struct Rel5Grid {
  int nx, nh, nvp, nve, order;
  int64_t n;               // cells
  int64_t sy, sp, se, sv;  // strides of y, psi, vE, vP (x stride is 1)
  double extent, dx, dphi, dvp, dve;
  double vp_lo, ve_lo, acc_p, acc_e, curv_p, curv_e;
};

// Device-side reduction words of one handle.
struct Rel5Stats {
  unsigned long long residual;  // bits of a non-negative double
  unsigned long long increase;  // bits of a non-negative double
  unsigned int nonfinite;       // set when an update is not finite
  unsigned int pad;
};

struct Rel5Stage {
  const float *src;  // stage input
  float *dst;        // stage output (stage 2: also holds the step's old V)
  float *arrival;    // first-crossing time, NaN until the cell enters
  const double *sn, *cs;   // sin/cos of the heading axis, double
  const float *snf, *csf;  // the same, rounded to float
  double dt, t;            // step size and the step's start time
  Rel5Stats *stats;
};

// Fast path: float32 local arithmetic.  blend = 0 for stage 1 (or the only
// stage of RK1), 1 for the RK2 averaging stage.
cudaError_t rel5_stage_f32(const Rel5Grid &g, const Rel5Stage &s, int blend,
                           cudaStream_t stream);

// Exact path: double local arithmetic in the reference's operation order,
// built without contraction so it reproduces native_relative.cpp bit for bit.
cudaError_t rel5_stage_f64(const Rel5Grid &g, const Rel5Stage &s, int blend,
                           cudaStream_t stream);

// Broadcast a (y, x) plane of initial values over every (vP, vE, psi) and set
// arrival = start_time where the value is <= 0, NaN elsewhere.  With
// plane == nullptr the field is taken as already filled and only arrival is
// set.
cudaError_t rel5_init(const Rel5Grid &g, const float *plane, float *field,
                      float *arrival, float start_time, cudaStream_t stream);

}  // namespace pe
