/* Test infrastructure (the oracle library): a check, in the host's IEEE
 * double arithmetic, of the division used by the GPU exact stage
 * (csrc/div_rn.cuh, rn::div_const): a / b for b > 0 as the product
 * a * r with r = RN(1/b), corrected once through an FMA (Markstein's
 * correction theorem: with q0 = RN(a r) and the exact residual
 * a - b q0, RN(q0 + residual * r) = RN(a / b) when nothing underflows or
 * overflows), zeros and far-out dividends taking the division itself.
 * po_div_const_check draws n dividends of the kinds the stage divides
 * (differences and second differences of floats, random doubles over a
 * wide exponent range, signed zeros, subnormals) and counts those whose
 * quotient differs from a / b in any bit.  The product never calls it. */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

static double div_const(double a, double b, double r) {
  const double m = fabs(a);
  if (!(m >= 0x1p-900 && m <= 0x1p+900)) return a == 0.0 ? a * r : a / b;
  const double q0 = a * r;
  const double rho = fma(-q0, b, a);
  return rho == 0.0 ? q0 : fma(rho, r, q0);
}

static float div_constf(float a, float b, float r) {
  const float m = fabsf(a);
  if (!(m >= 0x1p-80f && m <= 0x1p+100f)) return a == 0.f ? a * r : a / b;
  const float q0 = a * r;
  const float rho = fmaf(-q0, b, a);
  return rho == 0.f ? q0 : fmaf(rho, r, q0);
}

static uint64_t next(uint64_t *s) {
  *s ^= *s << 13;
  *s ^= *s >> 7;
  *s ^= *s << 17;
  return *s;
}

static double unit(uint64_t *s) { return (next(s) >> 11) * (1.0 / 9007199254740992.0); }

long long po_div_const_check(double b, long long n, unsigned long long seed) {
  uint64_t s = seed ? seed : 88172645463325252ull;
  const double r = 1.0 / b;
  long long bad = 0;
  for (long long i = 0; i < n; i++) {
    double a;
    switch (i % 5) {
      case 0: a = (unit(&s) * 2 - 1) * ldexp(1.0, (int)(next(&s) % 60) - 50); break;
      case 1: {
        const float f1 = (float)(unit(&s) * 2 - 1), f0 = (float)(unit(&s) * 2 - 1);
        a = (double)f1 - (double)f0;
        break;
      }
      case 2: {
        const float f = (float)(unit(&s) * 4 - 2), g = (float)(unit(&s) * 4 - 2);
        const float h = (float)(unit(&s) * 4 - 2);
        a = (double)g - 2 * (double)f + (double)h;
        break;
      }
      case 3: {
        uint64_t bits = next(&s);
        bits = (bits & 0x800FFFFFFFFFFFFFull) |
               ((uint64_t)(1023 + (int)(next(&s) % 40) - 20) << 52);
        memcpy(&a, &bits, sizeof a);
        break;
      }
      default: {
        const double z[6] = {-0.0, 0.0, -1e-300, 1e-300, -ldexp(1.0, -1070), ldexp(1.0, -1070)};
        a = z[next(&s) % 6];
      }
    }
    const double q1 = a / b, q2 = div_const(a, b, r);
    if (memcmp(&q1, &q2, sizeof q1) != 0) bad++;
  }
  return bad;
}

/* The same for the float32 stages (8D and 6D): b and 1/b in float. */
long long po_div_const_checkf(float b, long long n, unsigned long long seed) {
  uint64_t s = seed ? seed : 88172645463325252ull;
  const float r = 1.0f / b;
  long long bad = 0;
  for (long long i = 0; i < n; i++) {
    float a;
    switch (i % 5) {
      case 0: a = (float)((unit(&s) * 2 - 1) * ldexp(1.0, (int)(next(&s) % 60) - 50)); break;
      case 1: a = (float)(unit(&s) * 2 - 1) - (float)(unit(&s) * 2 - 1); break;
      case 2: {
        const float f = (float)(unit(&s) * 4 - 2), g = (float)(unit(&s) * 4 - 2);
        const float h = (float)(unit(&s) * 4 - 2);
        a = g - 2 * f + h;
        break;
      }
      case 3: {
        uint32_t bits = (uint32_t)next(&s);
        bits = (bits & 0x807FFFFFu) | ((uint32_t)(127 + (int)(next(&s) % 60) - 30) << 23);
        memcpy(&a, &bits, sizeof a);
        break;
      }
      default: {
        const float z[8] = {-0.0f, 0.0f, 1e-40f, -1e-40f, 1e-30f, -3e-25f, ldexpf(1.0f, -149),
                            -ldexpf(1.0f, -140)};
        a = z[next(&s) % 8];
      }
    }
    const float q1 = a / b, q2 = div_constf(a, b, r);
    if (memcmp(&q1, &q2, sizeof q1) != 0) bad++;
  }
  return bad;
}
