// Dense 8D ENO/Lax-Friedrichs stage kernel, shared by the exact variant
// (world8d_exact.cu, compiled with -fmad=false: float32 arithmetic in the
// order of native_world.cpp:32-74 and :261-314, bit for bit the reference
// executable's) and the fast variant (world8d_fast.cu: reciprocal spacings
// and multiply-add contraction, equal to float rounding).
//
// One thread per cell: blockIdx.y walks the pursuer block (xP, yP, thP, vP),
// the x dimension the evader block (xE, yE, thE, vE).
#pragma once
#include "div_rn.cuh"
#include "world8d.cuh"

namespace pe {
namespace w8 {

// Value beyond a non-periodic end: the end value pushed away from zero by
// the end difference, once per missing node (native_world.cpp:44-58).
__device__ __forceinline__ float ghost(const float *__restrict__ v, int64_t j,
                                       int64_t stride, int pos, int n,
                                       int offset, bool periodic) {
  int q = pos + offset;
  if (periodic) {  // |offset| <= 2 <= n: one wrap at most
    q = q < 0 ? q + n : (q >= n ? q - n : q);
    return v[j + (int64_t)(q - pos) * stride];
  }
  if (q < 0) {
    const int64_t edge = j - (int64_t)pos * stride;
    const float a = v[edge], b = v[edge + stride];
    return a + (-q) * fabsf(b - a) * ((a > 0) - (a < 0));
  }
  if (q >= n) {
    const int64_t edge = j + (int64_t)(n - 1 - pos) * stride;
    const float a = v[edge], b = v[edge - stride];
    return a + (q - n + 1) * fabsf(a - b) * ((a > 0) - (a < 0));
  }
  return v[j + (int64_t)offset * stride];
}

// Difference quotients: the reference divides (exact variant, through
// div_const, bit for bit); the fast variant multiplies by the reciprocal
// spacing.
template <bool FAST>
__device__ __forceinline__ float quot(float d, float h, float ih) {
  return FAST ? d * ih : rn::div_const(d, h, ih);
}

template <bool FAST>
__device__ __forceinline__ void slopes(const float *__restrict__ v, int64_t j,
                                       int64_t stride, int pos, int n, float h, float ih,
                                       float ihh_rn, bool periodic, bool inward, int order,
                                       float &lo, float &hi) {
  if (inward && pos == 0) {
    lo = hi = quot<FAST>(v[j + stride] - v[j], h, ih);
    return;
  }
  if (inward && pos == n - 1) {
    lo = hi = quot<FAST>(v[j] - v[j - stride], h, ih);
    return;
  }
  const float f = v[j];
  const float fm = ghost(v, j, stride, pos, n, -1, periodic);
  const float fp = ghost(v, j, stride, pos, n, 1, periodic);
  lo = quot<FAST>(f - fm, h, ih);
  hi = quot<FAST>(fp - f, h, ih);
  if (order == 2) {
    // exact variant: 1/(h*h) rounded to nearest; fast variant: (1/h)^2
    const float hh = h * h, ihh = FAST ? ih * ih : ihh_rn;
    const float dc = quot<FAST>(fp - 2 * f + fm, hh, ihh);
    const float dl = inward && pos < 2
                         ? dc
                         : quot<FAST>(f - 2 * fm + ghost(v, j, stride, pos, n, -2, periodic),
                                      hh, ihh);
    const float dr = inward && pos + 2 >= n
                         ? dc
                         : quot<FAST>(ghost(v, j, stride, pos, n, 2, periodic) - 2 * fp + f,
                                      hh, ihh);
    lo += .5f * h * (fabsf(dl) <= fabsf(dc) ? dl : dc);
    hi -= .5f * h * (fabsf(dc) <= fabsf(dr) ? dc : dr);
  }
}

template <bool FAST>
// 6 CTAs of 256 threads per SM: the stage waits on its stencil loads, and
// more warps hide them (7.45 against 7.74 ms per RK2 step at config 4)
__global__ void __launch_bounds__(256, 6)
    world8_stage_kernel(const World8Grid g, const World8Stage s) {
  __shared__ float warp_max[8];
  const int inner = g.shape[4] * g.shape[5] * g.shape[6] * g.shape[7];
  const int outer = g.shape[0] * g.shape[1] * g.shape[2] * g.shape[3];
  const int e_cell = blockIdx.x * blockDim.x + threadIdx.x;
  float change_max = 0.f;
  bool bad = false;
  for (int o = blockIdx.y; o < outer; o += gridDim.y) {
    if (e_cell < inner) {
      const int64_t j = (int64_t)o * inner + e_cell;
      int q[8];
      {
        int rest = o;
        q[3] = rest % g.shape[3];
        rest /= g.shape[3];
        q[2] = rest % g.shape[2];
        rest /= g.shape[2];
        q[1] = rest % g.shape[1];
        q[0] = rest / g.shape[1];
        int e = e_cell;
        q[7] = e % g.shape[7];
        e /= g.shape[7];
        q[6] = e % g.shape[6];
        e /= g.shape[6];
        q[5] = e % g.shape[5];
        q[4] = e / g.shape[5];
      }
      const float vp = s.pv[q[3]];
      const float palo = q[3] == 0 ? 0 : -g.ap;
      const float pahi = q[3] == g.np - 1 ? 0 : g.ap;
      const float fpx = vp * s.cs[q[2]], fpy = vp * s.sn[q[2]];
      const float wp = fabsf(vp) * g.kp;
      const float ve = s.ev[q[7]], we = fabsf(ve) * g.ke;
      const float ealo = q[7] == 0 ? 0 : -g.ae;
      const float eahi = q[7] == g.ne - 1 ? 0 : g.ae;
      const float flow[8] = {fpx, fpy, 0, 0, ve * s.cs[q[6]], ve * s.sn[q[6]], 0, 0};
      float grad[8], H = 0, diss = 0;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        float lm, rp;
        slopes<FAST>(s.src, j, g.stride[k], q[k], g.shape[k], g.spacing[k],
                     g.inv_spacing[k], g.inv_spacing_sq[k], k == 2 || k == 6,
                     g.linear_speed && (k == 3 || k == 7), g.order, lm, rp);
        grad[k] = .5f * (lm + rp);
        const float alpha = k == 2   ? wp
                            : k == 3 ? g.ap
                            : k == 6 ? we
                            : k == 7 ? g.ae
                                     : fabsf(flow[k]);
        H += flow[k] * grad[k];
        diss += .5f * alpha * (rp - lm);
      }
      const float p_lo_term = palo * grad[3], p_hi_term = pahi * grad[3];
      const float e_lo_term = ealo * grad[7], e_hi_term = eahi * grad[7];
      H += -wp * fabsf(grad[2]) + we * fabsf(grad[6]) +
           (p_hi_term < p_lo_term ? p_hi_term : p_lo_term) +
           (e_lo_term < e_hi_term ? e_hi_term : e_lo_term);
      float value = s.src[j] + s.dt * (H + diss);
      if (s.base) value = .5f * (s.base[j] + value);
      if (g.order == 1 || s.base) {
        const float previous = s.base ? s.base[j] : s.src[j];
        // std::max(std::min(value, previous), avoid)
        const float tube = previous < value ? previous : value;
        float avoid = -INFINITY;
        if (g.avoid_mode == 1) {
          const float ax = fabsf(s.x[q[0]]), ay = fabsf(s.x[q[1]]);
          avoid = (ax < ay ? ay : ax) - g.arena + 1e-6f;
        } else if (g.avoid_mode == 2) {
          avoid = -s.p_clear[(q[0] * g.n + q[1]) * g.nh + q[2]] + 1e-6f;
        }
        value = tube < avoid ? avoid : tube;
        if (previous > 0 && value <= 0 && isnan(s.arrival[j]))
          s.arrival[j] = (float)s.tau + s.dt * previous / (previous - value);
        change_max = fmaxf(change_max, fabsf(value - previous));
      }
      if (!isfinite(value)) bad = true;
      s.dst[j] = value;
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&s.stats->nonfinite, 1u);
  for (int off = 16; off > 0; off >>= 1)
    change_max = fmaxf(change_max, __shfl_xor_sync(0xffffffffu, change_max, off));
  if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = change_max;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, warp_max[w]);
    if (m > 0.f)
      atomicMax(&s.stats->residual, (unsigned long long)__double_as_longlong((double)m));
  }
}

template <bool FAST>
cudaError_t launch_stage(const World8Grid &g, const World8Stage &s, cudaStream_t stream) {
  const int64_t inner = (int64_t)g.shape[4] * g.shape[5] * g.shape[6] * g.shape[7];
  const int64_t outer = g.cells / inner;
  const dim3 grid((unsigned)((inner + 255) / 256),
                  (unsigned)(outer < 65535 ? outer : 65535));
  world8_stage_kernel<FAST><<<grid, 256, 0, stream>>>(g, s);
  return cudaGetLastError();
}

}  // namespace w8
}  // namespace pe
