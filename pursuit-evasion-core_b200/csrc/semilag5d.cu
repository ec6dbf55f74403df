// Relative 5D semi-Lagrangian min-max backup on the GPU (float32).
//
// Semantics (restated from the reference's building blocks; the reference
// itself has no 5D semi-Lagrangian solver):
//   successor   exact held-command arcs, reversible/model.py:86-183, with
//               the per-(speed, action) arc data tabulated on the host in
//               double (SLPursuerArc, SLEvaderArc, SLEvaderMove);
//   actions     product([-A,0,A],[-K,0,K]), reversible/controllers.py:19-27;
//   min-max     min over pursuer actions of max over evader actions, the
//               minimum starting at the current value (tube minimum,
//               local_game/grid_game.py:218-230) or, for the minimum-time
//               functional, u' = 0 inside the capture disk and
//               (1 - b) + b * min max u(s') outside;
//   interpolate multilinear over [vP, vE, psi, y, x], periodic psi,
//               reversible/relative_table.py:76-102, linear beyond the
//               position box;
//   ties        pursuer: smallest (|k|, |a|, index) among values within 1e-7
//               of the minimum (controllers.py:122-126); evader: first in
//               the neutral-first order of map_game_policy.py:12-18.
// One thread per cell; the block's (vP, vE, psi) arc tables sit in shared
// memory.  In value-only mode a pursuer action whose running evader maximum
// already reaches the best value so far is abandoned (grid_game.py:226):
// the value is unchanged by it.
#include "semilag5d.cuh"

namespace pe {
namespace {

__device__ __constant__ int kEvaderOrder[9] = {4, 1, 7, 3, 5, 0, 2, 6, 8};

// Lower node and weight of a non-periodic axis (clamped node, extrapolated
// weight).
__device__ __forceinline__ void locate_clamped(float f, int n, int &j, float &w) {
  int k = __float2int_rd(f);
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  j = k;
  w = f - (float)k;
}

template <bool POLICY>
__global__ void __launch_bounds__(128)
    sl_backup_kernel(const SLGrid g, const SLBackup b) {
  __shared__ SLPursuerArc sp[9];
  __shared__ SLEvaderArc se[9];
  __shared__ SLEvaderMove sm[9];
  __shared__ float warp_max[4];
  const int ip = blockIdx.y;
  const int ie = blockIdx.z % g.nve, iv = blockIdx.z / g.nve;
  if (threadIdx.x < 9) {
    sp[threadIdx.x] = b.parc[iv * 9 + threadIdx.x];
    se[threadIdx.x] = b.earc[ie * 9 + threadIdx.x];
    sm[threadIdx.x] = b.emove[((int64_t)ip * g.nve + ie) * 9 + threadIdx.x];
  }
  __syncthreads();
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  float change = 0.f;
  bool bad = false;
  if (cell < g.nx * g.nx) {
    const int ix = cell % g.nx, iy = cell / g.nx;
    const float x = fmaf((float)ix, g.dx, -g.extent);
    const float y = fmaf((float)iy, g.dx, -g.extent);
    const int64_t j = (int64_t)blockIdx.z * g.se + (int64_t)ip * g.sp + cell;
    const float *__restrict__ V = b.src;
    const float current = V[j];
    float best = (g.mode == SL_TUBE) ? current : INFINITY;
    float worst_of[9];
    int e_of[9];
    for (int up = 0; up < 9; up++) {
      const SLPursuerArc pa = sp[up];
      // pursuer speed corner(s)
      int jv;
      float wv;
      locate_clamped(pa.fv, g.nvp, jv, wv);
      float worst = -INFINITY;
      float vals[POLICY ? 9 : 1];
      for (int ue = 0; ue < 9; ue++) {
        const SLEvaderArc ea = se[ue];
        const SLEvaderMove em = sm[ue];
        const float dxp = x + em.ex - pa.px, dyp = y + em.ey - pa.py;
        const float xr = fmaf(pa.c, dxp, pa.s * dyp);
        const float yr = fmaf(pa.c, dyp, -pa.s * dxp);
        int jx, jy, je;
        float wx, wy, we;
        locate_clamped((xr + g.extent) * g.ihx, g.nx, jx, wx);
        locate_clamped((yr + g.extent) * g.ihx, g.nx, jy, wy);
        locate_clamped(ea.fv, g.nve, je, we);
        const float fpsi = (float)ip + (ea.turn_idx - pa.turn_idx);
        const float fl = floorf(fpsi);
        const float wp = fpsi - fl;
        int jp = (int)fl % g.nh;
        jp += jp < 0 ? g.nh : 0;
        const int jp1 = jp + 1 == g.nh ? 0 : jp + 1;
        float value = 0.f;
#pragma unroll
        for (int bv = 0; bv < 2; bv++) {
          const float w_v = bv ? wv : 1.f - wv;
          if (w_v == 0.f) continue;
#pragma unroll
          for (int be = 0; be < 2; be++) {
            const float w_e = be ? we : 1.f - we;
            if (w_e == 0.f) continue;
            const int64_t speed_base = (int64_t)(jv + bv) * g.sv + (int64_t)(je + be) * g.se;
            float acc_p = 0.f;
#pragma unroll
            for (int bp = 0; bp < 2; bp++) {
              const int64_t pb = speed_base + (int64_t)(bp ? jp1 : jp) * g.sp +
                                 (int64_t)jy * g.sy + jx;
              const float v00 = __ldg(V + pb), v01 = __ldg(V + pb + 1);
              const float v10 = __ldg(V + pb + g.sy), v11 = __ldg(V + pb + g.sy + 1);
              const float r0 = fmaf(wx, v01 - v00, v00);
              const float r1 = fmaf(wx, v11 - v10, v10);
              const float plane = fmaf(wy, r1 - r0, r0);
              acc_p = bp ? fmaf(wp, plane - acc_p, acc_p) : plane;
            }
            value = fmaf(w_v * w_e, acc_p, value);
          }
        }
        if (g.mode == SL_MINTIME) value = fminf(fmaxf(value, 0.f), 1.f);
        if (POLICY) vals[ue] = value;
        worst = fmaxf(worst, value);
        if (!POLICY && worst >= best) break;  // cannot lower the minimum
      }
      if (POLICY) {
        worst_of[up] = worst;
        int pick = kEvaderOrder[0];
#pragma unroll
        for (int r = 0; r < 9; r++)
          if (vals[kEvaderOrder[r]] >= worst - 1e-7f) {
            pick = kEvaderOrder[r];
            break;
          }
        e_of[up] = pick;
      }
      best = fminf(best, worst);
    }
    float out;
    if (g.mode == SL_TUBE) {
      out = best;
    } else {
      const float d = hypotf(x, y) - g.radius;  // capture test of this cell
      out = d <= 0.f ? 0.f : fmaf(g.beta, best, 1.f - g.beta);
    }
    if (POLICY) {
      float lo = INFINITY;
      for (int up = 0; up < 9; up++) lo = fminf(lo, worst_of[up]);
      int pick = 0, key = 1 << 30;
      for (int up = 0; up < 9; up++) {
        if (worst_of[up] > lo + 1e-7f) continue;
        const int k = ((abs(up % 3 - 1) * 2 + abs(up / 3 - 1)) << 4) + up;
        if (k < key) {
          key = k;
          pick = up;
        }
      }
      b.policy_p[j] = (uint8_t)pick;
      b.policy_e[j] = (uint8_t)e_of[pick];
    }
    if (!isfinite(out)) bad = true;
    b.dst[j] = out;
    change = fabsf(out - current);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&b.stats->nonfinite, 1u);
  for (int off = 16; off > 0; off >>= 1)
    change = fmaxf(change, __shfl_xor_sync(0xffffffffu, change, off));
  if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = change;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, warp_max[w]);
    if (m > 0.f)
      atomicMax(&b.stats->residual, (unsigned long long)__double_as_longlong((double)m));
  }
}

__global__ void sl_init_kernel(const float *plane, float *field, int64_t n,
                               int plane_size) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    field[j] = plane[j % plane_size];
}

}  // namespace

cudaError_t sl_backup(const SLGrid &g, const SLBackup &b, cudaStream_t stream) {
  const int threads = 128;
  const dim3 grid((g.nx * g.nx + threads - 1) / threads, g.nh, g.nvp * g.nve);
  if (b.policy_p)
    sl_backup_kernel<true><<<grid, threads, 0, stream>>>(g, b);
  else
    sl_backup_kernel<false><<<grid, threads, 0, stream>>>(g, b);
  return cudaGetLastError();
}

__global__ void sl_arrival_kernel(const float *__restrict__ prev, const float *__restrict__ cur,
                                  float *__restrict__ arrival, int64_t n, double t, double dt) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const float p = prev[j], v = cur[j];
    if (p > 0.f && v <= 0.f && isnan(arrival[j]))
      arrival[j] = (float)(t + dt * (double)p / ((double)p - (double)v));
  }
}

cudaError_t sl_arrival(const SLGrid &g, const float *prev, const float *cur, float *arrival,
                       double t, double dt, cudaStream_t stream) {
  sl_arrival_kernel<<<148 * 8, 256, 0, stream>>>(prev, cur, arrival, g.n, t, dt);
  return cudaGetLastError();
}

__global__ void sl_arrival_start_kernel(const float *__restrict__ cur,
                                        float *__restrict__ arrival, int64_t n, float t) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    arrival[j] = cur[j] <= 0.f ? t : __int_as_float(0x7fc00000);
}

cudaError_t sl_arrival_start(const SLGrid &g, const float *cur, float *arrival,
                             double start_time, cudaStream_t stream) {
  sl_arrival_start_kernel<<<148 * 8, 256, 0, stream>>>(cur, arrival, g.n, (float)start_time);
  return cudaGetLastError();
}

cudaError_t sl_init(const SLGrid &g, const float *plane, float *field,
                    cudaStream_t stream) {
  sl_init_kernel<<<148 * 16, 256, 0, stream>>>(plane, field, g.n, g.nx * g.nx);
  return cudaGetLastError();
}

}  // namespace pe
