// Relative 5D ENO/LF stage, fast variant: float32 storage and float32 local
// arithmetic.  Same scheme as native_relative.cpp:38-172 (ENO1/ENO2 slopes,
// Isaacs Hamiltonian, local Lax-Friedrichs dissipation, RK1/RK2, tube
// minimum through min(0, H), first-crossing arrival), with the algebra
// arranged for fewer instructions:
//   * second differences are kept unscaled (h^2 * D2), the slope is formed as
//     (first difference +- 0.5 * selected second difference) / h, which is
//     the reference's dm + 0.5*h*D2 rewritten;
//   * 1/h is precomputed, divisions become multiplies.
// Results agree with the double-local reference to float rounding; the
// exact variant (relative5d_exact.cu) is the bit-for-bit path.
#include "relative5d.cuh"

namespace pe {
namespace {

struct SlopesF {
  float lo, hi;
};

template <int ORDER>
__device__ __forceinline__ SlopesF eno_axis_f(const float *__restrict__ s,
                                              int64_t j, int64_t stride,
                                              int pos, int n, float ih,
                                              bool periodic, float v) {
  SlopesF r;
  if (!periodic && pos == 0) {
    r.lo = r.hi = (__ldg(s + j + stride) - v) * ih;
    return r;
  }
  if (!periodic && pos == n - 1) {
    r.lo = r.hi = (v - __ldg(s + j - stride)) * ih;
    return r;
  }
  const int64_t wrap = (int64_t)n * stride;
  const int64_t om1 = (periodic && pos < 1) ? wrap - stride : -stride;
  const int64_t op1 = (periodic && pos + 1 >= n) ? stride - wrap : stride;
  const float vm = __ldg(s + j + om1), vp = __ldg(s + j + op1);
  const float d_lo = v - vm, d_hi = vp - v;
  if (ORDER == 1) {
    r.lo = d_lo * ih;
    r.hi = d_hi * ih;
    return r;
  }
  const float c2 = d_hi - d_lo;
  float l2 = c2, r2 = c2;
  if (periodic || pos >= 2) {
    const int64_t om2 = (periodic && pos < 2) ? wrap - 2 * stride : -2 * stride;
    l2 = d_lo - (vm - __ldg(s + j + om2));
  }
  if (periodic || pos + 2 < n) {
    const int64_t op2 =
        (periodic && pos + 2 >= n) ? 2 * stride - wrap : 2 * stride;
    r2 = (__ldg(s + j + op2) - vp) - d_hi;
  }
  const float sel_lo = fabsf(l2) < fabsf(c2) ? l2 : c2;
  const float sel_hi = fabsf(c2) < fabsf(r2) ? c2 : r2;
  r.lo = fmaf(0.5f, sel_lo, d_lo) * ih;
  r.hi = fmaf(-0.5f, sel_hi, d_hi) * ih;
  return r;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *word,
                                                  double value) {
  if (value > 0) atomicMax(word, (unsigned long long)__double_as_longlong(value));
}

template <int ORDER, int BLEND>
__global__ void __launch_bounds__(256)
    rel5_stage_fast_kernel(const Rel5Grid g, const Rel5Stage s) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  const int plane = g.nx * g.nx;
  float residual = 0.f;
  if (cell < plane) {
    const int ix = cell % g.nx, iy = cell / g.nx;
    const int ip = blockIdx.y;
    const int ie = blockIdx.z % g.nve, iv = blockIdx.z / g.nve;
    const int64_t j = (int64_t)blockIdx.z * g.se + (int64_t)ip * g.sp + cell;
    const float *__restrict__ src = s.src;
    const float ihx = (float)(1.0 / g.dx), ihp = (float)(1.0 / g.dphi);
    const float ihv = (float)(1.0 / g.dvp), ihe = (float)(1.0 / g.dve);

    const float x = (float)(-g.extent + ix * g.dx);
    const float y = (float)(-g.extent + iy * g.dx);
    const float vp = (float)(g.vp_lo + iv * g.dvp);
    const float ve = (float)(g.ve_lo + ie * g.dve);
    const float wp = fabsf(vp) * (float)g.curv_p;
    const float we = fabsf(ve) * (float)g.curv_e;
    const float bx = fmaf(ve, s.csf[ip], -vp), by = ve * s.snf[ip];
    const float ap = (float)g.acc_p, ae = (float)g.acc_e;

    const float v = __ldg(src + j);
    const SlopesF sx = eno_axis_f<ORDER>(src, j, 1, ix, g.nx, ihx, false, v);
    const SlopesF sy = eno_axis_f<ORDER>(src, j, g.sy, iy, g.nx, ihx, false, v);
    const SlopesF sp = eno_axis_f<ORDER>(src, j, g.sp, ip, g.nh, ihp, true, v);
    const SlopesF sv = eno_axis_f<ORDER>(src, j, g.sv, iv, g.nvp, ihv, false, v);
    const SlopesF se = eno_axis_f<ORDER>(src, j, g.se, ie, g.nve, ihe, false, v);

    const float gx = 0.5f * (sx.lo + sx.hi), gy = 0.5f * (sy.lo + sy.hi);
    const float gp = 0.5f * (sp.lo + sp.hi), gv = 0.5f * (sv.lo + sv.hi);
    const float ge = 0.5f * (se.lo + se.hi);
    // Pursuer picks the acceleration minimising ap*gv (0 if it points out of
    // the speed range), the evader maximises ae*ge likewise.
    const float p_term = iv == 0           ? fminf(0.f, ap * gv)
                         : iv == g.nvp - 1 ? fminf(-ap * gv, 0.f)
                                           : -ap * fabsf(gv);
    const float e_term = ie == 0           ? fmaxf(0.f, ae * ge)
                         : ie == g.nve - 1 ? fmaxf(-ae * ge, 0.f)
                                           : ae * fabsf(ge);
    float H = fmaf(bx, gx, by * gy);
    H = fmaf(-wp, fabsf(fmaf(y, gx, -fmaf(x, gy, gp))), H);
    H = fmaf(we, fabsf(gp), H);
    H += p_term + e_term;
    float diss = (fabsf(bx) + wp * fabsf(y)) * (sx.hi - sx.lo);
    diss = fmaf(fabsf(by) + wp * fabsf(x), sy.hi - sy.lo, diss);
    diss = fmaf(wp + we, sp.hi - sp.lo, diss);
    diss = fmaf(ap, sv.hi - sv.lo, diss);
    diss = fmaf(ae, se.hi - se.lo, diss);
    H = fmaf(0.5f, diss, H);

    const float dt = (float)s.dt;
    const float prev = BLEND ? s.dst[j] : v;
    float value = fmaf(dt, fminf(H, 0.f), v);
    if (BLEND) value = 0.5f * (prev + value);
    if (!isfinite(value)) {
      atomicOr(&s.stats->nonfinite, 1u);
    } else {
      s.dst[j] = value;
      if (BLEND || ORDER == 1) {
        residual = fabsf(value - prev);
        if (prev > 0.f && value <= 0.f && isnan(s.arrival[j]))
          s.arrival[j] = (float)(s.t + s.dt * (double)prev /
                                           ((double)prev - (double)value));
      }
    }
  }
  if (BLEND || ORDER == 1) {
    // Block max of |V_new - V_old| (each cell's change rounded to float),
    // folded into the handle's double reduction word by one atomic per block.
    for (int off = 16; off > 0; off >>= 1)
      residual = fmaxf(residual, __shfl_xor_sync(0xffffffffu, residual, off));
    __shared__ float warp_max[8];
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = residual;
    __syncthreads();
    if (threadIdx.x == 0) {
      float m = warp_max[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, warp_max[w]);
      atomic_max_nonneg(&s.stats->residual, (double)m);
    }
  }
}

__global__ void rel5_init_kernel(const float *__restrict__ plane,
                                 float *__restrict__ field,
                                 float *__restrict__ arrival, int64_t n,
                                 int plane_size, float start_time) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const float v = plane ? plane[j % plane_size] : field[j];
    if (plane) field[j] = v;
    arrival[j] = v <= 0.f ? start_time : __int_as_float(0x7fc00000);
  }
}

}  // namespace

cudaError_t rel5_stage_f32(const Rel5Grid &g, const Rel5Stage &s, int blend,
                           cudaStream_t stream) {
  const int threads = 256;
  const dim3 grid((g.nx * g.nx + threads - 1) / threads, g.nh, g.nvp * g.nve);
  if (g.order == 1)
    rel5_stage_fast_kernel<1, 0><<<grid, threads, 0, stream>>>(g, s);
  else if (blend)
    rel5_stage_fast_kernel<2, 1><<<grid, threads, 0, stream>>>(g, s);
  else
    rel5_stage_fast_kernel<2, 0><<<grid, threads, 0, stream>>>(g, s);
  return cudaGetLastError();
}

cudaError_t rel5_init(const Rel5Grid &g, const float *plane, float *field,
                      float *arrival, float start_time, cudaStream_t stream) {
  const int threads = 256;
  int64_t blocks = (g.n + threads - 1) / threads;
  if (blocks > 148 * 64) blocks = 148 * 64;
  rel5_init_kernel<<<(unsigned)blocks, threads, 0, stream>>>(
      plane, field, arrival, g.n, g.nx * g.nx, start_time);
  return cudaGetLastError();
}

}  // namespace pe
