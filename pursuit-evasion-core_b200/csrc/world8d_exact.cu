// Dense 8D ENO/Lax-Friedrichs stage on the GPU, float32 arithmetic in the
// order of native_world.cpp:32-74 (slopes) and :261-314 (stage).  This file
// is compiled with -fmad=false so that no multiply-add is fused: every stored
// float equals the reference CPU executable's bit for bit.
//
// One thread per cell: blockIdx.y walks the pursuer block
// (xP, yP, thP, vP), the x dimension the evader block (xE, yE, thE, vE).
#include "world8d.cuh"

namespace pe {
namespace {

// Value beyond a non-periodic end: the end value pushed away from zero by
// the end difference, once per missing node (native_world.cpp:44-58).
__device__ __forceinline__ float ghost(const float *__restrict__ v, int64_t j,
                                       int64_t stride, int pos, int n,
                                       int offset, bool periodic) {
  int q = pos + offset;
  if (periodic) {
    q = (q % n + n) % n;
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

__device__ __forceinline__ void slopes(const float *__restrict__ v, int64_t j,
                                       int64_t stride, int pos, int n, float h,
                                       bool periodic, bool inward, int order,
                                       float &lo, float &hi) {
  if (inward && pos == 0) {
    lo = hi = (v[j + stride] - v[j]) / h;
    return;
  }
  if (inward && pos == n - 1) {
    lo = hi = (v[j] - v[j - stride]) / h;
    return;
  }
  const float f = v[j];
  const float fm = ghost(v, j, stride, pos, n, -1, periodic);
  const float fp = ghost(v, j, stride, pos, n, 1, periodic);
  lo = (f - fm) / h;
  hi = (fp - f) / h;
  if (order == 2) {
    const float dc = (fp - 2 * f + fm) / (h * h);
    const float dl = inward && pos < 2
                         ? dc
                         : (f - 2 * fm + ghost(v, j, stride, pos, n, -2, periodic)) / (h * h);
    const float dr = inward && pos + 2 >= n
                         ? dc
                         : (ghost(v, j, stride, pos, n, 2, periodic) - 2 * fp + f) / (h * h);
    lo += .5f * h * (fabsf(dl) <= fabsf(dc) ? dl : dc);
    hi -= .5f * h * (fabsf(dc) <= fabsf(dr) ? dc : dr);
  }
}

__global__ void __launch_bounds__(256)
    world8_stage_kernel(const World8Grid g, const World8Stage s) {
  __shared__ float warp_max[8];
  const int64_t inner = (int64_t)g.shape[4] * g.shape[5] * g.shape[6] * g.shape[7];
  const int64_t outer = g.cells / inner;
  const int e_cell = blockIdx.x * blockDim.x + threadIdx.x;
  float change_max = 0.f;
  bool bad = false;
  for (int64_t o = blockIdx.y; o < outer; o += gridDim.y) {
    if (e_cell < inner) {
      const int64_t j = o * inner + e_cell;
      int q[8];
      {
        int64_t rest = o;
        q[3] = (int)(rest % g.shape[3]);
        rest /= g.shape[3];
        q[2] = (int)(rest % g.shape[2]);
        rest /= g.shape[2];
        q[1] = (int)(rest % g.shape[1]);
        q[0] = (int)(rest / g.shape[1]);
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
        slopes(s.src, j, g.stride[k], q[k], g.shape[k], g.spacing[k],
               k == 2 || k == 6, g.linear_speed && (k == 3 || k == 7), g.order,
               lm, rp);
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

// Separating-axis contact value of two oriented rectangles (double), in the
// order of the oracle's po_rect_separation.
__global__ void world8_contact_kernel(World8Grid g, const double *cs,
                                      const double *sn, const double *cdiff,
                                      const double *sdiff, double p_len,
                                      double p_wid, double e_len, double e_wid,
                                      double dxd, float *field,
                                      float *arrival) {
  const int64_t poses = g.cells / g.shape[7];  // speeds do not enter
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < poses;
       p += (int64_t)gridDim.x * blockDim.x) {
    // p enumerates [xP, yP, thP, vP, xE, yE, thE]
    int64_t rest = p;
    const int the = (int)(rest % g.shape[6]);
    rest /= g.shape[6];
    const int ye = (int)(rest % g.shape[5]);
    rest /= g.shape[5];
    const int xe = (int)(rest % g.shape[4]);
    rest /= g.shape[4];
    rest /= g.shape[3];  // vP
    const int thp = (int)(rest % g.shape[2]);
    rest /= g.shape[2];
    const int yp = (int)(rest % g.shape[1]);
    const int xp = (int)(rest / g.shape[1]);
    const double ext = (double)g.extent;
    const double px = -ext + xp * dxd, py = -ext + yp * dxd;
    const double ex = -ext + xe * dxd, ey = -ext + ye * dxd;
    const double d0 = ex - px, d1 = ey - py;
    // cos/sin of (thE - thP), tabulated on the host with the C library
    const double ca = fabs(cdiff[the * g.nh + thp]), sa = fabs(sdiff[the * g.nh + thp]);
    double best = -INFINITY;
    const int hk[2] = {thp, the};
    const double own_l[2] = {p_len, e_len}, own_w[2] = {p_wid, e_wid};
    const double oth_l[2] = {e_len, p_len}, oth_w[2] = {e_wid, p_wid};
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const double c = cs[hk[k]], s_ = sn[hk[k]];
      const double x = d0 * c + d1 * s_;
      const double y = -d0 * s_ + d1 * c;
      const double gx = fabs(x) - own_l[k] / 2 - (oth_l[k] * ca + oth_w[k] * sa) / 2;
      const double gy = fabs(y) - own_w[k] / 2 - (oth_l[k] * sa + oth_w[k] * ca) / 2;
      if (gx > best) best = gx;
      if (gy > best) best = gy;
    }
    const float value = (float)best;
    for (int v = 0; v < g.shape[7]; v++) {
      field[p * g.shape[7] + v] = value;
      arrival[p * g.shape[7] + v] = value <= 0 ? 0.f : __int_as_float(0x7fc00000);
    }
  }
}

__global__ void world8_square_kernel(World8Grid g, const float *x, float radius,
                                     float *field, float *arrival) {
  const int64_t block = (int64_t)g.shape[6] * g.shape[7];
  const int64_t blocks = g.cells / block;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < blocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    int64_t rest = b;
    const int ye = (int)(rest % g.shape[5]);
    rest /= g.shape[5];
    const int xe = (int)(rest % g.shape[4]);
    rest /= g.shape[4];
    rest /= g.shape[3];
    rest /= g.shape[2];
    const int yp = (int)(rest % g.shape[1]);
    const int xp = (int)(rest / g.shape[1]);
    const float capture = hypotf(x[xp] - x[xe], x[yp] - x[ye]) - radius;
    const float axe = fabsf(x[xe]), aye = fabsf(x[ye]);
    const float e_fault = g.arena - (axe < aye ? aye : axe);
    const float target = e_fault < capture ? e_fault : capture;
    const float axp = fabsf(x[xp]), ayp = fabsf(x[yp]);
    const float avoid = (axp < ayp ? ayp : axp) - g.arena + 1e-6f;
    const float initial = target < avoid ? avoid : target;
    for (int64_t k = 0; k < block; k++) {
      field[b * block + k] = initial;
      arrival[b * block + k] = initial <= 0 ? 0.f : __int_as_float(0x7fc00000);
    }
  }
}

__global__ void world8_arrival_kernel(int64_t n, const float *field,
                                      float *arrival, float start) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    arrival[j] = field[j] <= 0 ? start : __int_as_float(0x7fc00000);
}

}  // namespace

cudaError_t world8_stage(const World8Grid &g, const World8Stage &s,
                         cudaStream_t stream) {
  const int64_t inner = (int64_t)g.shape[4] * g.shape[5] * g.shape[6] * g.shape[7];
  const int64_t outer = g.cells / inner;
  const dim3 grid((unsigned)((inner + 255) / 256),
                  (unsigned)(outer < 65535 ? outer : 65535));
  world8_stage_kernel<<<grid, 256, 0, stream>>>(g, s);
  return cudaGetLastError();
}

cudaError_t world8_init_contact(const World8Grid &g, const double *cs,
                                const double *sn, const double *cdiff,
                                const double *sdiff, double p_len, double p_wid,
                                double e_len, double e_wid, float *field,
                                float *arrival, cudaStream_t stream) {
  const double dxd = 2 * (double)g.extent / (g.n - 1);
  world8_contact_kernel<<<148 * 8, 256, 0, stream>>>(g, cs, sn, cdiff, sdiff, p_len,
                                                     p_wid, e_len, e_wid, dxd, field,
                                                     arrival);
  return cudaGetLastError();
}

cudaError_t world8_init_square(const World8Grid &g, const float *x,
                               float radius, float *field, float *arrival,
                               cudaStream_t stream) {
  world8_square_kernel<<<148 * 8, 256, 0, stream>>>(g, x, radius, field, arrival);
  return cudaGetLastError();
}

cudaError_t world8_init_arrival(const World8Grid &g, const float *field,
                                float *arrival, float start,
                                cudaStream_t stream) {
  world8_arrival_kernel<<<148 * 8, 256, 0, stream>>>(g.cells, field, arrival, start);
  return cudaGetLastError();
}

}  // namespace pe
