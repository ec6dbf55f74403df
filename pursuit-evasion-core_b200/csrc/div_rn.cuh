// Division by a grid spacing in the exact (reference-order) stages, with the
// bits of the IEEE division: a / b rounded to nearest for b > 0, given
// r = 1/b rounded to nearest, by Markstein's correction of the product a * r
// (P. Markstein, "IA-64 and Elementary Functions", 2000; Muller et al.,
// "Handbook of Floating-Point Arithmetic", the correction theorem for
// division).  With q0 = RN(a r), the residual a - b q0 is exact through an
// FMA, and RN(q0 + residual * r) equals RN(a / b) whenever nothing
// underflows or overflows.  A zero residual means q0 is already exact (and
// keeps the sign of a zero a); dividends outside a range far from
// underflow and overflow (zeros, NaN, subnormal or huge values) take the
// division itself.  One multiply and two FMAs instead of a full division.
// The host check oracle/divcheck.c and the GPU parity tests pin it.
#pragma once
#include <cuda_runtime.h>

namespace pe {
namespace rn {

__device__ __forceinline__ double div_const(double a, double b, double r) {
  const double m = fabs(a);
  if (!(m >= 0x1p-900 && m <= 0x1p+900)) return a == 0.0 ? a * r : a / b;
  const double q0 = a * r;
  const double rho = fma(-q0, b, a);
  return rho == 0.0 ? q0 : fma(rho, r, q0);
}

__device__ __forceinline__ float div_const(float a, float b, float r) {
  const float m = fabsf(a);
  if (!(m >= 0x1p-80f && m <= 0x1p+100f)) return a == 0.f ? a * r : a / b;
  const float q0 = a * r;
  const float rho = fmaf(-q0, b, a);
  return rho == 0.f ? q0 : fmaf(rho, r, q0);
}

}  // namespace rn
}  // namespace pe
