// Legacy six-dimensional square game (src/pursuit_evasion/dp/native_square.cpp):
// one stage of the ENO1/ENO2 Lax-Friedrichs RK1/RK2 update in float32, in
// the reference's operation order.  This translation unit is compiled
// without multiply-add contraction (-fmad=false) and with IEEE divisions,
// so every stage equals the reference executable's bit for bit.
//
// Storage [xP, yP, thP, xE, yE, thE], thE fastest.  One thread per cell:
// blockIdx.y walks the pursuer block (xP, yP, thP), the x dimension the
// evader block (xE, yE, thE).
#include "div_rn.cuh"
#include "square6d.cuh"

namespace pe {
namespace {

// Value at `offset` nodes along an axis: periodic wrap, or beyond a
// non-periodic end the end value pushed away from zero by the end
// difference once per missing node (native_square.cpp:33-49).
__device__ __forceinline__ float at(const float *__restrict__ v, int64_t j, int64_t stride,
                                    int pos, int n, int offset, bool periodic) {
  int q = pos + offset;
  if (periodic) {
    q = q < 0 ? q + n : (q >= n ? q - n : q);  // |offset| <= 2 < n
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

// Backward / forward ENO slopes (native_square.cpp:50-61).
// rh, rhh: 1/h and 1/(h*h) rounded to nearest; the divisions keep the
// reference's bits (rn::div_const).
__device__ __forceinline__ void slopes(const float *__restrict__ v, int64_t j, int64_t stride,
                                       int pos, int n, float h, float rh, float rhh,
                                       bool periodic, int order, float &left, float &right) {
  const float f = v[j], fm = at(v, j, stride, pos, n, -1, periodic),
              fp = at(v, j, stride, pos, n, 1, periodic);
  left = rn::div_const(f - fm, h, rh);
  right = rn::div_const(fp - f, h, rh);
  if (order == 2) {
    const float hh = h * h;
    const float dl = rn::div_const(f - 2 * fm + at(v, j, stride, pos, n, -2, periodic), hh, rhh);
    const float dc = rn::div_const(fp - 2 * f + fm, hh, rhh);
    const float dr = rn::div_const(at(v, j, stride, pos, n, 2, periodic) - 2 * fp + f, hh, rhh);
    const float a = fabsf(dl) <= fabsf(dc) ? dl : dc;
    const float b = fabsf(dc) <= fabsf(dr) ? dc : dr;
    left += .5f * h * a;
    right -= .5f * h * b;
  }
}

__global__ void __launch_bounds__(256)
    square6_stage_kernel(const Square6Grid g, const Square6Stage s) {
  __shared__ float warp_max[8];
  const int inner = g.n * g.n * g.nh, outer = inner;
  const int e_cell = blockIdx.x * blockDim.x + threadIdx.x;
  float change_max = 0.f;
  bool bad = false;
  for (int o = blockIdx.y; o < outer; o += gridDim.y) {
    if (e_cell < inner) {
      const int64_t j = (int64_t)o * inner + e_cell;
      int q[6];
      q[5] = e_cell % g.nh;
      q[4] = (e_cell / g.nh) % g.n;
      q[3] = e_cell / (g.nh * g.n);
      q[2] = o % g.nh;
      q[1] = (o / g.nh) % g.n;
      q[0] = o / (g.nh * g.n);
      // native_square.cpp:150-167
      const float f[6] = {g.vp * s.cs[q[2]], g.vp * s.sn[q[2]], 0,
                          g.ve * s.cs[q[5]], g.ve * s.sn[q[5]], 0};
      float gr[6], diss = 0, H = 0;
#pragma unroll
      for (int k = 0; k < 6; k++) {
        float lm, rp;
        const bool periodic = k == 2 || k == 5;
        slopes(s.src, j, g.stride[k], q[k], periodic ? g.nh : g.n, periodic ? g.dh : g.dx,
               periodic ? g.rdh : g.rdx, periodic ? g.rdh2 : g.rdx2, periodic, g.order, lm,
               rp);
        gr[k] = (lm + rp) * .5f;
        const float alpha = k == 2 ? g.wp : k == 5 ? g.we : fabsf(f[k]);
        diss += alpha * (rp - lm) * .5f;
        H += f[k] * gr[k];
      }
      H += -g.wp * fabsf(gr[2]) + g.we * fabsf(gr[5]);
      float value = s.src[j] + s.dt * (H + diss);
      if (s.base) value = .5f * (s.base[j] + value);
      if (g.order == 1 || s.base) {
        const float previous = s.base ? s.base[j] : s.src[j];
        const float ax = fabsf(s.x[q[0]]), ay = fabsf(s.x[q[1]]);
        const float avoid = (ax < ay ? ay : ax) - g.arena + 1e-6f;
        // std::max(std::min(value, previous), avoid)
        const float tube = previous < value ? previous : value;
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

// The initial field: one value per (xP, yP, xE, yE) (`block`, computed on
// the host), repeated over both headings; arrival 0 where <= 0, else NaN.
__global__ void square6_init_kernel(const Square6Grid g, const float *__restrict__ block,
                                    float *__restrict__ field, float *__restrict__ arrival) {
  const int64_t n = g.cells;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = j / g.nh;  // drop thE
    const int ye = (int)(r % g.n), xe = (int)(r / g.n % g.n);
    const int64_t p = r / ((int64_t)g.n * g.n) / g.nh;  // drop thP: (xP, yP)
    const float v = block[(p * g.n + xe) * g.n + ye];
    field[j] = v;
    arrival[j] = v <= 0 ? 0.f : __int_as_float(0x7fc00000);
  }
}

}  // namespace

cudaError_t square6_stage(const Square6Grid &g, const Square6Stage &s, cudaStream_t stream) {
  const int inner = g.n * g.n * g.nh;
  const dim3 grid((unsigned)((inner + 255) / 256), (unsigned)(inner < 65535 ? inner : 65535));
  square6_stage_kernel<<<grid, 256, 0, stream>>>(g, s);
  return cudaGetLastError();
}

cudaError_t square6_init(const Square6Grid &g, const float *block, float *field,
                         float *arrival, cudaStream_t stream) {
  square6_init_kernel<<<148 * 16, 256, 0, stream>>>(g, block, field, arrival);
  return cudaGetLastError();
}

}  // namespace pe
