// Dense 8D ENO/Lax-Friedrichs stage, fast variant (float32, multiply-add
// contraction, reciprocal spacings): the update of native_world.cpp:261-314
// equal to the exact stage up to float rounding and the ENO2 selections that
// rounding can flip.
//
// Layout [xP, yP, thP, vP | xE, yE, thE, vE]: the cells of one pursuer pose
// (xP, yP, thP, vP) form a contiguous "evader block" (11*11*9*7 = 7,623 cells
// on the 8D contact grid).  A CTA walks the pursuer poses o = blockIdx.x,
// blockIdx.x + gridDim.x, ...; for each it stages the evader block in shared
// memory (cp.async, double-buffered so the next block loads while this one
// computes).  The four evader-axis stencils read shared memory; the four
// pursuer-axis stencils read the same cell of the neighbouring blocks, one
// coalesced load per neighbour, from L2.
//
// Ghost values beyond a non-periodic end (native_world.cpp:44-58) are rebuilt
// from the clamped 5-value window: every ghost the reference forms is the end
// value pushed by the end difference, and both lie inside the window.  The
// Hamiltonian's linear flow terms and their Lax-Friedrichs dissipation fold
// into upwind weights: v*g + |v|/2 (hi - lo) = min(v,0) lo + max(v,0) hi.
// Evader blocks too large for shared memory use the thread-per-cell kernel
// of world8d_stage.cuh.
#include <cstdio>

#include "relative5d_eno_f32.cuh"
#include "world8d_stage.cuh"

namespace pe {
namespace {

using eno32::add2;
using eno32::f2;
using eno32::sub2;

constexpr int kThreads = 256;
constexpr int kMaxBlockBytes = 96 * 1024;  // per buffer; two buffers per CTA
constexpr size_t kMaxColumnBytes = 112 * 1024;  // column kernel: two CTAs per SM

// e / d as __umulhi(e, m), m = ceil(2^32 / d): exact for e * (m*d - 2^32) <
// 2^32, which holds for e < 2^24 and d < 256 and, in general, for e < 2^32/d.
struct Divisor {
  uint32_t m;
  int d;
};

Divisor make_divisor(int d) {
  return {(uint32_t)((((uint64_t)1 << 32) + (uint64_t)d - 1) / (uint64_t)d), d};
}

__device__ __forceinline__ int split(int e, Divisor v, int &rem) {
  const int q = (int)__umulhi((uint32_t)e, v.m);
  rem = e - q * v.d;
  return q;
}

struct FastW8Args {
  World8Grid g;
  World8Stage s;
  Divisor d7, d6, d5;
  int inner, outer;
};

enum AxisKind { kExtrapolated = 0, kPeriodic = 1, kInward = 2 };

// a + m |b - a| sign(a): the reference's value beyond an end (a: end node,
// b: the node next to it, m: nodes beyond the end).
__device__ __forceinline__ float ghost_value(float a, float b, float m) {
  const float sgn = a > 0.f ? 1.f : (a < 0.f ? -1.f : 0.f);
  return fmaf(m * fabsf(b - a), sgn, a);
}

// Unscaled backward / forward ENO slopes (times the spacing) of a cell at
// position p of an axis of n nodes, from its clamped (or wrapped) window.
template <int ORDER>
__device__ __forceinline__ void axis_slopes(float m2, float m1, float f, float p1,
                                            float p2, int p, int n, int kind,
                                            float &dlo, float &dhi) {
  if (kind == kExtrapolated && (p < 2 || p + 2 >= n)) {
    if (p == 0) {
      m1 = ghost_value(f, p1, 1.f);
      m2 = ghost_value(f, p1, 2.f);
    } else if (p == 1) {
      m2 = ghost_value(m1, f, 1.f);
    }
    if (p == n - 1) {
      p1 = ghost_value(f, m1, 1.f);
      p2 = ghost_value(f, m1, 2.f);
    } else if (p == n - 2) {
      p2 = ghost_value(p1, f, 1.f);
    }
  }
  dlo = f - m1;
  dhi = p1 - f;
  if (ORDER == 2) {
    // Second-difference numerators in the reference's form (fp - 2f + fm):
    // 2f is exact, so they round as the reference's do and the ENO choices
    // below break exact ties (frequent on the piecewise-linear contact field)
    // the same way; dividing both sides by h^2 keeps the comparison.
    const float c = (p1 - 2.f * f) + m1;
    float l = (f - 2.f * m1) + m2;
    float r = (p2 - 2.f * p1) + f;
    if (kind == kInward) {
      if (p < 2) l = c;
      if (p + 2 >= n) r = c;
    }
    // ties pick the outer difference on the low side and the centred one on
    // the high side (native_world.cpp:70-71)
    const float el = fabsf(l) <= fabsf(c) ? l : c;
    const float er = fabsf(c) <= fabsf(r) ? c : r;
    dlo = fmaf(0.5f, el, dlo);
    dhi = fmaf(-0.5f, er, dhi);
  }
  if (kind == kInward) {
    if (p == 0) dlo = dhi = p1 - f;
    if (p == n - 1) dlo = dhi = f - m1;
  }
}

// The same slopes for two independent cells at the same position p of the
// axis, in packed FP32 (__ffma2_rn / __fadd2_rn round each element as the
// scalar operation does); the ENO selections and the end-node ghosts are
// taken element by element.
template <int ORDER>
__device__ __forceinline__ void axis_slopes2(float2 m2, float2 m1, float2 f, float2 p1,
                                             float2 p2, int p, int n, int kind, float2 &dlo,
                                             float2 &dhi) {
  if (kind == kExtrapolated && (p < 2 || p + 2 >= n)) {
    if (p == 0) {
      m1 = make_float2(ghost_value(f.x, p1.x, 1.f), ghost_value(f.y, p1.y, 1.f));
      m2 = make_float2(ghost_value(f.x, p1.x, 2.f), ghost_value(f.y, p1.y, 2.f));
    } else if (p == 1) {
      m2 = make_float2(ghost_value(m1.x, f.x, 1.f), ghost_value(m1.y, f.y, 1.f));
    }
    if (p == n - 1) {
      p1 = make_float2(ghost_value(f.x, m1.x, 1.f), ghost_value(f.y, m1.y, 1.f));
      p2 = make_float2(ghost_value(f.x, m1.x, 2.f), ghost_value(f.y, m1.y, 2.f));
    } else if (p == n - 2) {
      p2 = make_float2(ghost_value(p1.x, f.x, 1.f), ghost_value(p1.y, f.y, 1.f));
    }
  }
  dlo = sub2(f, m1);
  dhi = sub2(p1, f);
  if (ORDER == 2) {
    // (fp - 2f) + fm with 2f exact, as the scalar form
    const float2 c = add2(__ffma2_rn(f, f2(-2.f), p1), m1);
    float2 l = add2(__ffma2_rn(m1, f2(-2.f), f), m2);
    float2 r = add2(__ffma2_rn(p1, f2(-2.f), p2), f);
    if (kind == kInward) {
      if (p < 2) l = c;
      if (p + 2 >= n) r = c;
    }
    const float2 el = make_float2(fabsf(l.x) <= fabsf(c.x) ? l.x : c.x,
                                  fabsf(l.y) <= fabsf(c.y) ? l.y : c.y);
    const float2 er = make_float2(fabsf(c.x) <= fabsf(r.x) ? c.x : r.x,
                                  fabsf(c.y) <= fabsf(r.y) ? c.y : r.y);
    dlo = __ffma2_rn(f2(0.5f), el, dlo);
    dhi = __ffma2_rn(f2(-0.5f), er, dhi);
  }
  if (kind == kInward) {
    if (p == 0) dlo = dhi = sub2(p1, f);
    if (p == n - 1) dlo = dhi = sub2(f, m1);
  }
}

// Window offsets (in cells) of positions p-2, p-1, p+1, p+2 along an axis of
// stride s: clamped to the ends, or wrapped when periodic.
__device__ __forceinline__ void window_offsets(int p, int n, int s, bool periodic,
                                               int &om2, int &om1, int &op1, int &op2) {
  if (periodic) {
    om1 = p > 0 ? -s : (n - 1) * s;
    om2 = p > 1 ? -2 * s : (n - 2) * s;
    op1 = p < n - 1 ? s : -(n - 1) * s;
    op2 = p < n - 2 ? 2 * s : -(n - 2) * s;
  } else {
    om1 = p > 0 ? -s : 0;
    om2 = p > 1 ? -2 * s : om1;
    op1 = p < n - 1 ? s : 0;
    op2 = p < n - 2 ? 2 * s : op1;
  }
}

__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_one() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <int ORDER>
__global__ void __launch_bounds__(kThreads)
    world8_block_kernel(const FastW8Args a) {
  extern __shared__ __align__(16) float blocks[];  // [2][inner]
  __shared__ float warp_max[kThreads / 32];
  const World8Grid &g = a.g;
  const World8Stage &s = a.s;
  const int inner = a.inner, tid = threadIdx.x;
  const int kind_speed = g.linear_speed ? kInward : kExtrapolated;
  // evader strides inside a block and pursuer strides (whole blocks)
  const int s7 = 1, s6 = g.shape[7], s5 = g.shape[6] * s6, s4 = g.shape[5] * s5;
  const float ih[8] = {g.inv_spacing[0], g.inv_spacing[1], g.inv_spacing[2],
                       g.inv_spacing[3], g.inv_spacing[4], g.inv_spacing[5],
                       g.inv_spacing[6], g.inv_spacing[7]};
  float change_max = 0.f;
  bool bad = false;

  auto stage_block = [&](int o, float *dst) {
    const float *src = s.src + (int64_t)o * inner;
    for (int e = tid; e < inner; e += kThreads) cp_async4(dst + e, src + e);
  };

  int buf = 0;
  if ((int)blockIdx.x < a.outer) stage_block(blockIdx.x, blocks);
  cp_async_commit();
  for (int o = blockIdx.x; o < a.outer; o += gridDim.x, buf ^= 1) {
    const int next = o + gridDim.x;
    if (next < a.outer) stage_block(next, blocks + (buf ^ 1) * inner);
    cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
    const float *blk = blocks + buf * inner;

    // pursuer pose (uniform over the CTA)
    int qp[4];
    {
      int rest = o;
      qp[3] = rest % g.shape[3];
      rest /= g.shape[3];
      qp[2] = rest % g.shape[2];
      rest /= g.shape[2];
      qp[1] = rest % g.shape[1];
      qp[0] = rest / g.shape[1];
    }
    const float vp = __ldg(s.pv + qp[3]);
    const float fpx = vp * __ldg(s.cs + qp[2]), fpy = vp * __ldg(s.sn + qp[2]);
    const float wp = fabsf(vp) * g.kp;
    const float palo = qp[3] == 0 ? 0.f : -g.ap;
    const float pahi = qp[3] == g.np - 1 ? 0.f : g.ap;
    // upwind weights of the pursuer position axes (unscaled slopes)
    const float wx_lo = fminf(fpx, 0.f) * ih[0], wx_hi = fmaxf(fpx, 0.f) * ih[0];
    const float wy_lo = fminf(fpy, 0.f) * ih[1], wy_hi = fmaxf(fpy, 0.f) * ih[1];
    float avoid = -INFINITY;
    if (g.avoid_mode == 1) {
      const float ax = fabsf(__ldg(s.x + qp[0])), ay = fabsf(__ldg(s.x + qp[1]));
      avoid = (ax < ay ? ay : ax) - g.arena + 1e-6f;
    } else if (g.avoid_mode == 2) {
      avoid = -__ldg(s.p_clear + (qp[0] * g.n + qp[1]) * g.nh + qp[2]) + 1e-6f;
    }
    // neighbour offsets along the pursuer axes, in cells
    int64_t poff[4][4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int om2, om1, op1, op2;
      window_offsets(qp[k], g.shape[k], 1, k == 2, om2, om1, op1, op2);
      const int64_t st = g.stride[k];
      poff[k][0] = om2 * st;
      poff[k][1] = om1 * st;
      poff[k][2] = op1 * st;
      poff[k][3] = op2 * st;
    }
    const int64_t j0 = (int64_t)o * inner;
    const float *__restrict__ src_o = s.src + j0;
    // The pursuer-axis values (the same evader cell in the 16 neighbouring
    // blocks, from L2 or HBM) of a thread's next cell are loaded while its
    // current cell is computed, so their latency overlaps the arithmetic.
    float ahead[16];
    auto load_pursuer = [&](int e, float v[16]) {
#pragma unroll
      for (int k = 0; k < 4; k++)
#pragma unroll
        for (int m = 0; m < 4; m++) v[4 * k + m] = __ldg(src_o + poff[k][m] + e);
    };
    if (tid < inner) load_pursuer(tid, ahead);

    for (int e = tid; e < inner; e += kThreads) {
      float nbv[16];
#pragma unroll
      for (int i = 0; i < 16; i++) nbv[i] = ahead[i];
      if (e + kThreads < inner) load_pursuer(e + kThreads, ahead);
      int q7, q6, q5;
      int t = split(e, a.d7, q7);
      t = split(t, a.d6, q6);
      const int q4 = split(t, a.d5, q5);
      const float f = blk[e];
      float dlo[8], dhi[8];
      // pursuer axes: the same evader cell in the neighbouring blocks
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int kind = k == 2 ? kPeriodic : (k == 3 ? kind_speed : kExtrapolated);
        axis_slopes<ORDER>(nbv[4 * k], nbv[4 * k + 1], f, nbv[4 * k + 2], nbv[4 * k + 3],
                           qp[k], g.shape[k], kind, dlo[k], dhi[k]);
      }
      // evader axes: shared memory
      const int qe[4] = {q4, q5, q6, q7};
      const int se[4] = {s4, s5, s6, s7};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        int om2, om1, op1, op2;
        window_offsets(qe[k], g.shape[4 + k], se[k], k == 2, om2, om1, op1, op2);
        const int kind = k == 2 ? kPeriodic : (k == 3 ? kind_speed : kExtrapolated);
        axis_slopes<ORDER>(blk[e + om2], blk[e + om1], f, blk[e + op1], blk[e + op2],
                           qe[k], g.shape[4 + k], kind, dlo[4 + k], dhi[4 + k]);
      }
      const float ve = __ldg(s.ev + q7);
      const float fex = ve * __ldg(s.cs + q6), fey = ve * __ldg(s.sn + q6);
      const float we = fabsf(ve) * g.ke;
      const float ealo = q7 == 0 ? 0.f : -g.ae;
      const float eahi = q7 == g.ne - 1 ? 0.f : g.ae;
      // linear flow axes with their dissipation: upwind weights
      float total = fmaf(wx_lo, dlo[0], wx_hi * dhi[0]);
      total = fmaf(wy_lo, dlo[1], fmaf(wy_hi, dhi[1], total));
      total = fmaf(fminf(fex, 0.f) * ih[4], dlo[4], fmaf(fmaxf(fex, 0.f) * ih[4], dhi[4], total));
      total = fmaf(fminf(fey, 0.f) * ih[5], dlo[5], fmaf(fmaxf(fey, 0.f) * ih[5], dhi[5], total));
      // headings: -wp |g_thP| + we |g_thE| and their dissipation
      const float g2 = 0.5f * ih[2] * (dlo[2] + dhi[2]);
      const float g6 = 0.5f * ih[6] * (dlo[6] + dhi[6]);
      total = fmaf(-wp, fabsf(g2), total);
      total = fmaf(we, fabsf(g6), total);
      float diss = wp * ih[2] * (dhi[2] - dlo[2]);
      diss = fmaf(we * ih[6], dhi[6] - dlo[6], diss);
      // speeds: bounded accelerations
      const float g3 = 0.5f * ih[3] * (dlo[3] + dhi[3]);
      const float g7 = 0.5f * ih[7] * (dlo[7] + dhi[7]);
      total += fminf(palo * g3, pahi * g3) + fmaxf(ealo * g7, eahi * g7);
      diss = fmaf(g.ap * ih[3], dhi[3] - dlo[3], diss);
      diss = fmaf(g.ae * ih[7], dhi[7] - dlo[7], diss);
      total = fmaf(0.5f, diss, total);

      const int64_t j = j0 + e;
      float value = fmaf(s.dt, total, f);
      if (s.base) value = 0.5f * (__ldg(s.base + j) + value);
      if (g.order == 1 || s.base) {
        const float previous = s.base ? __ldg(s.base + j) : f;
        const float tube = previous < value ? previous : value;
        value = tube < avoid ? avoid : tube;
        if (previous > 0.f && value <= 0.f && isnan(s.arrival[j]))
          s.arrival[j] = (float)s.tau + s.dt * previous / (previous - value);
        change_max = fmaxf(change_max, fabsf(value - previous));
      }
      bad |= !isfinite(value);
      s.dst[j] = value;
    }
    __syncthreads();  // this buffer is refilled two poses later
  }
  asm volatile("cp.async.wait_all;" ::: "memory");

  if (__syncthreads_or(bad) && tid == 0) atomicOr(&s.stats->nonfinite, 1u);
  for (int off = 16; off > 0; off >>= 1)
    change_max = fmaxf(change_max, __shfl_xor_sync(0xffffffffu, change_max, off));
  if ((tid & 31) == 0) warp_max[tid >> 5] = change_max;
  __syncthreads();
  if (tid == 0) {
    float m = 0.f;
    for (int w = 0; w < kThreads / 32; w++) m = fmaxf(m, warp_max[w]);
    if (m > 0.f)
      atomicMax(&s.stats->residual, (unsigned long long)__double_as_longlong((double)m));
  }
}

template <int ORDER>
cudaError_t launch_block(const FastW8Args &a, size_t smem, cudaStream_t stream) {
  static size_t configured = 0;
  static int resident = 0;
  if (configured != smem || resident == 0) {
    cudaError_t e = cudaFuncSetAttribute(world8_block_kernel<ORDER>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, world8_block_kernel<ORDER>,
                                                      kThreads, smem);
    if (e != cudaSuccess) return e;
    if (resident < 1) return cudaErrorInvalidConfiguration;
    configured = smem;
  }
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = a.outer < sms * resident ? a.outer : sms * resident;
  world8_block_kernel<ORDER><<<blocks, kThreads, smem, stream>>>(a);
  return cudaGetLastError();
}


// ------------------------------------------------------------ column kernel
// The same stage with the work of a pursuer pose split in two passes, so
// that no per-cell position or end-rule logic is left:
//   B (a thread per vE column, i.e. per (xE, yE, thE)): the four evader-axis
//     stencils from the staged block.  vE runs along the column in registers
//     with its end rules at compile-time positions (NE nodes); thE wraps by
//     per-column offsets; xE and yE read a copy of the block padded by two
//     ghost rows on each side, filled once per pose with the reference's
//     extrapolated values (native_world.cpp:44-58: the value beyond an end
//     is the end node pushed by m times the end difference), so every
//     position takes the interior formula.  The evader terms and their
//     dissipation go to part[cell] in shared memory;
//   A + C (a thread per cell, consecutive cells on consecutive lanes): the
//     four pursuer-axis stencils from the 16 neighbouring blocks (coalesced
//     L2 loads of the next cell issued while the current one computes; the
//     pose, hence every pursuer end rule, is uniform over the CTA), then the
//     update, RK2 average, tube, avoid floor, arrival and residual with
//     coalesced loads and stores.
// The block of the next pose is requested by cp.async (a warp per (xE, yE)
// row) as soon as pass B is done, and lands during pass A + C.  Sums are
// taken evader part first, so results differ from world8_block_kernel's by
// float rounding.
constexpr int kColThreads = 256;
constexpr int kCBatch = 8;  // cells per thread whose update loads are issued together

struct ColW8Args {
  World8Grid g;
  World8Stage s;
  int inner, outer, ncols;
  Divisor dnh, dn;
};

// shared memory floats: padded block [n+4][n+4][nh][NE] + partial sums [inner]
inline size_t column_smem_bytes(const World8Grid &g) {
  const size_t row = (size_t)g.nh * g.shape[7];
  return sizeof(float) * row * ((size_t)(g.n + 4) * (g.n + 4) + (size_t)g.n * g.n);
}

template <int ORDER, int NE, int SKIND>
__global__ void __launch_bounds__(kColThreads, 2)
    world8_column_kernel(const ColW8Args a) {
  extern __shared__ __align__(16) float sm[];
  __shared__ float warp_max[kColThreads / 32];
  const World8Grid &g = a.g;
  const World8Stage &s = a.s;
  const int inner = a.inner, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = kColThreads / 32;
  const int n = g.n, nh = g.nh;
  const int rowlen = nh * NE;                  // one (xE, yE) row: all (thE, vE)
  const int sy = rowlen, sx = (n + 4) * rowlen;  // padded strides of yE and xE
  float *pad = sm;                             // [n+4][n+4][nh][NE]
  float *part = sm + (n + 4) * sx;             // [inner]
  const float ih[8] = {g.inv_spacing[0], g.inv_spacing[1], g.inv_spacing[2],
                       g.inv_spacing[3], g.inv_spacing[4], g.inv_spacing[5],
                       g.inv_spacing[6], g.inv_spacing[7]};
  float change_max = 0.f;
  bool bad = false;

  // the block of pose o into the padded interior, a warp per (xE, yE) row
  auto stage_block = [&](int o) {
    const float *src = s.src + (int64_t)o * inner;
    for (int r = warp; r < n * n; r += nwarps) {
      const int q4 = r / n, q5 = r - q4 * n;
      float *dst = pad + (q4 + 2) * sx + (q5 + 2) * sy;
      const float *row = src + r * rowlen;
      for (int j = lane; j < rowlen; j += 32) cp_async4(dst + j, row + j);
    }
  };
  // ghost rows beyond the xE and yE ends (needs the interior in place):
  // side 0-3 xE = -2, -1, n, n+1 at yE = idx; side 4-7 the same along yE at
  // xE = idx
  auto fill_ghosts = [&]() {
    for (int gr = warp; gr < 8 * n; gr += nwarps) {
      const int side = gr / n, idx = gr - side * n;
      const int q = side & 3;  // ghost position -2, -1, n, n+1
      const int pos = q < 2 ? q - 2 : n - 2 + q;
      const float m = q == 0 || q == 3 ? 2.f : 1.f;
      const int end = q < 2 ? 0 : n - 1, next = q < 2 ? 1 : n - 2;
      const int along = side < 4 ? sx : sy, across = side < 4 ? sy : sx;
      const float *row_a = pad + (end + 2) * along + (idx + 2) * across;
      const float *row_b = pad + (next + 2) * along + (idx + 2) * across;
      float *row_g = pad + (pos + 2) * along + (idx + 2) * across;
      for (int j = lane; j < rowlen; j += 32) row_g[j] = ghost_value(row_a[j], row_b[j], m);
    }
  };

  if ((int)blockIdx.x < a.outer) stage_block(blockIdx.x);
  cp_async_commit();
  for (int o = blockIdx.x; o < a.outer; o += gridDim.x) {
    // pursuer pose (uniform over the CTA)
    int qp[4];
    {
      int rest = o;
      qp[3] = rest % g.shape[3];
      rest /= g.shape[3];
      qp[2] = rest % g.shape[2];
      rest /= g.shape[2];
      qp[1] = rest % g.shape[1];
      qp[0] = rest / g.shape[1];
    }
    const float vp = __ldg(s.pv + qp[3]);
    const float fpx = vp * __ldg(s.cs + qp[2]), fpy = vp * __ldg(s.sn + qp[2]);
    const float wp = fabsf(vp) * g.kp;
    const float palo = qp[3] == 0 ? 0.f : -g.ap;
    const float pahi = qp[3] == g.np - 1 ? 0.f : g.ap;
    const float wx_lo = fminf(fpx, 0.f) * ih[0], wx_hi = fmaxf(fpx, 0.f) * ih[0];
    const float wy_lo = fminf(fpy, 0.f) * ih[1], wy_hi = fmaxf(fpy, 0.f) * ih[1];
    float avoid = -INFINITY;
    if (g.avoid_mode == 1) {
      const float ax = fabsf(__ldg(s.x + qp[0])), ay = fabsf(__ldg(s.x + qp[1]));
      avoid = (ax < ay ? ay : ax) - g.arena + 1e-6f;
    } else if (g.avoid_mode == 2) {
      avoid = -__ldg(s.p_clear + (qp[0] * g.n + qp[1]) * g.nh + qp[2]) + 1e-6f;
    }
    int poff[4][4];  // neighbour offsets along the pursuer axes, in cells
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int om2, om1, op1, op2;
      window_offsets(qp[k], g.shape[k], 1, k == 2, om2, om1, op1, op2);
      const int st = (int)g.stride[k];
      poff[k][0] = om2 * st;
      poff[k][1] = om1 * st;
      poff[k][2] = op1 * st;
      poff[k][3] = op2 * st;
    }
    const int64_t j0 = (int64_t)o * inner;
    const float *__restrict__ src_o = s.src + j0;

    // A: pursuer axes, a thread per cell (consecutive cells on consecutive
    // lanes), two cells at a time; the 2 x 17 loads (value and 16
    // pursuer-axis neighbours, from L2 or HBM) of the next two cells are
    // issued before the current two are computed
    auto load_cells = [&](int e, float (&buf)[2][17]) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = min(e + h * kColThreads, inner - 1);
        buf[h][16] = __ldg(src_o + c);
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
          for (int m = 0; m < 4; m++) buf[h][4 * k + m] = __ldg(src_o + poff[k][m] + c);
      }
    };
    // the two cells of a group in one packed pair (.x: e, .y: e + 256; the
    // second may lie past the block, computed from a clamped load and not
    // stored)
    auto pursuer_cells = [&](int e, const float (&buf)[2][17]) {
      auto at = [&](int i) { return make_float2(buf[0][i], buf[1][i]); };
      const float2 f = at(16);
      float2 dlo[4], dhi[4];
      axis_slopes2<ORDER>(at(0), at(1), f, at(2), at(3), qp[0], g.shape[0], kExtrapolated,
                          dlo[0], dhi[0]);
      axis_slopes2<ORDER>(at(4), at(5), f, at(6), at(7), qp[1], g.shape[1], kExtrapolated,
                          dlo[1], dhi[1]);
      axis_slopes2<ORDER>(at(8), at(9), f, at(10), at(11), qp[2], g.shape[2], kPeriodic,
                          dlo[2], dhi[2]);
      axis_slopes2<ORDER>(at(12), at(13), f, at(14), at(15), qp[3], g.shape[3], SKIND,
                          dlo[3], dhi[3]);
      float2 total = __ffma2_rn(f2(wx_lo), dlo[0], __fmul2_rn(f2(wx_hi), dhi[0]));
      total = __ffma2_rn(f2(wy_lo), dlo[1], __ffma2_rn(f2(wy_hi), dhi[1], total));
      const float2 g2 = __fmul2_rn(f2(0.5f * ih[2]), add2(dlo[2], dhi[2]));
      total = __ffma2_rn(f2(-wp), make_float2(fabsf(g2.x), fabsf(g2.y)), total);
      const float2 g3 = __fmul2_rn(f2(0.5f * ih[3]), add2(dlo[3], dhi[3]));
      total = add2(total, make_float2(fminf(palo * g3.x, pahi * g3.x),
                                      fminf(palo * g3.y, pahi * g3.y)));
      float2 diss = __fmul2_rn(f2(wp * ih[2]), sub2(dhi[2], dlo[2]));
      diss = __ffma2_rn(f2(g.ap * ih[3]), sub2(dhi[3], dlo[3]), diss);
      const float2 out = __ffma2_rn(f2(0.5f), diss, total);
      part[e] = out.x;
      if (e + kColThreads < inner) part[e + kColThreads] = out.y;
    };
    {
      constexpr int step = 2 * kColThreads;
      float bufA[2][17], bufB[2][17];
      if (tid < inner) load_cells(tid, bufA);
      for (int e = tid; e < inner; e += 2 * step) {
        if (e + step < inner) load_cells(e + step, bufB);
        pursuer_cells(e, bufA);
        if (e + step >= inner) break;
        if (e + 2 * step < inner) load_cells(e + 2 * step, bufA);
        pursuer_cells(e + step, bufB);
      }
    }
    cp_async_wait_all();
    __syncthreads();  // the block and every pursuer part are in place
    fill_ghosts();
    __syncthreads();

    // B: evader axes, a thread per vE column
    for (int c = tid; c < a.ncols; c += kColThreads) {
      int q6, q5;
      const int r = split(c, a.dnh, q6);
      const int q4 = split(r, a.dn, q5);
      const float *col = pad + (q4 + 2) * sx + (q5 + 2) * sy + q6 * NE;
      int om2, om1, op1, op2;
      window_offsets(q6, nh, NE, true, om2, om1, op1, op2);
      const float cs6 = __ldg(s.cs + q6), sn6 = __ldg(s.sn + q6);
      float vc[NE];
#pragma unroll
      for (int i = 0; i < NE; i++) vc[i] = col[i];
      float *pc = part + c * NE;
      // the clamped vE window of cell i: nodes i-2, i-1, i+1, i+2 (compile
      // time once unrolled)
      auto vw = [&](int i, int d) {
        return d == -2 ? vc[i > 1 ? i - 2 : (i > 0 ? i - 1 : i)]
             : d == -1 ? vc[i > 0 ? i - 1 : i]
             : d == 1  ? vc[i < NE - 1 ? i + 1 : i]
                       : vc[i < NE - 2 ? i + 2 : (i < NE - 1 ? i + 1 : i)];
      };
      // cell i alone
      auto evader_one = [&](int i) {
        const float f = vc[i];
        float dlo4, dhi4, dlo5, dhi5, dlo6, dhi6, dlo7, dhi7;
        // xE and yE: ghosts are in the padded block, every position is interior
        axis_slopes<ORDER>(col[i - 2 * sx], col[i - sx], f, col[i + sx], col[i + 2 * sx], 2, 5,
                           kPeriodic, dlo4, dhi4);
        axis_slopes<ORDER>(col[i - 2 * sy], col[i - sy], f, col[i + sy], col[i + 2 * sy], 2, 5,
                           kPeriodic, dlo5, dhi5);
        axis_slopes<ORDER>(col[i + om2], col[i + om1], f, col[i + op1], col[i + op2], 2, 5,
                           kPeriodic, dlo6, dhi6);
        // vE: the column's registers, compile-time end rules
        axis_slopes<ORDER>(vw(i, -2), vw(i, -1), f, vw(i, 1), vw(i, 2), i, NE, SKIND, dlo7,
                           dhi7);
        const float ve = __ldg(s.ev + i);
        const float fex = ve * cs6, fey = ve * sn6;
        const float we = fabsf(ve) * g.ke;
        const float ealo = i == 0 ? 0.f : -g.ae;
        const float eahi = i == NE - 1 ? 0.f : g.ae;
        float total = fmaf(fminf(fex, 0.f) * ih[4], dlo4, fmaxf(fex, 0.f) * ih[4] * dhi4);
        total = fmaf(fminf(fey, 0.f) * ih[5], dlo5, fmaf(fmaxf(fey, 0.f) * ih[5], dhi5, total));
        const float g6 = 0.5f * ih[6] * (dlo6 + dhi6);
        total = fmaf(we, fabsf(g6), total);
        const float g7 = 0.5f * ih[7] * (dlo7 + dhi7);
        total += fmaxf(ealo * g7, eahi * g7);
        float diss = we * ih[6] * (dhi6 - dlo6);
        diss = fmaf(g.ae * ih[7], dhi7 - dlo7, diss);
        pc[i] += fmaf(0.5f, diss, total);
      };
      // cells i and i+1 as one packed FP32 pair (vE slopes element by
      // element, for their compile-time end rules)
      auto evader_pair = [&](int i) {
        auto at = [&](int off) { return make_float2(col[i + off], col[i + 1 + off]); };
        const float2 f = make_float2(vc[i], vc[i + 1]);
        float2 dlo4, dhi4, dlo5, dhi5, dlo6, dhi6;
        axis_slopes2<ORDER>(at(-2 * sx), at(-sx), f, at(sx), at(2 * sx), 2, 5, kPeriodic, dlo4,
                            dhi4);
        axis_slopes2<ORDER>(at(-2 * sy), at(-sy), f, at(sy), at(2 * sy), 2, 5, kPeriodic, dlo5,
                            dhi5);
        axis_slopes2<ORDER>(at(om2), at(om1), f, at(op1), at(op2), 2, 5, kPeriodic, dlo6, dhi6);
        float alo, ahi, blo, bhi;
        axis_slopes<ORDER>(vw(i, -2), vw(i, -1), f.x, vw(i, 1), vw(i, 2), i, NE, SKIND, alo,
                           ahi);
        axis_slopes<ORDER>(vw(i + 1, -2), vw(i + 1, -1), f.y, vw(i + 1, 1), vw(i + 1, 2), i + 1,
                           NE, SKIND, blo, bhi);
        const float2 dlo7 = make_float2(alo, blo), dhi7 = make_float2(ahi, bhi);
        const float2 ve = make_float2(__ldg(s.ev + i), __ldg(s.ev + i + 1));
        const float2 fex = __fmul2_rn(ve, f2(cs6)), fey = __fmul2_rn(ve, f2(sn6));
        const float2 we = __fmul2_rn(make_float2(fabsf(ve.x), fabsf(ve.y)), f2(g.ke));
        const float2 ealo = make_float2(i == 0 ? 0.f : -g.ae, -g.ae);
        const float2 eahi = make_float2(g.ae, i + 1 == NE - 1 ? 0.f : g.ae);
        const float2 xlo = __fmul2_rn(make_float2(fminf(fex.x, 0.f), fminf(fex.y, 0.f)), f2(ih[4]));
        const float2 xhi = __fmul2_rn(make_float2(fmaxf(fex.x, 0.f), fmaxf(fex.y, 0.f)), f2(ih[4]));
        const float2 ylo = __fmul2_rn(make_float2(fminf(fey.x, 0.f), fminf(fey.y, 0.f)), f2(ih[5]));
        const float2 yhi = __fmul2_rn(make_float2(fmaxf(fey.x, 0.f), fmaxf(fey.y, 0.f)), f2(ih[5]));
        float2 total = __ffma2_rn(xlo, dlo4, __fmul2_rn(xhi, dhi4));
        total = __ffma2_rn(ylo, dlo5, __ffma2_rn(yhi, dhi5, total));
        const float2 g6 = __fmul2_rn(f2(0.5f * ih[6]), add2(dlo6, dhi6));
        total = __ffma2_rn(we, make_float2(fabsf(g6.x), fabsf(g6.y)), total);
        const float2 g7 = __fmul2_rn(f2(0.5f * ih[7]), add2(dlo7, dhi7));
        total = add2(total, make_float2(fmaxf(ealo.x * g7.x, eahi.x * g7.x),
                                        fmaxf(ealo.y * g7.y, eahi.y * g7.y)));
        float2 diss = __fmul2_rn(__fmul2_rn(we, f2(ih[6])), sub2(dhi6, dlo6));
        diss = __ffma2_rn(f2(g.ae * ih[7]), sub2(dhi7, dlo7), diss);
        const float2 out = __ffma2_rn(f2(0.5f), diss, total);
        pc[i] += out.x;
        pc[i + 1] += out.y;
      };
#pragma unroll
      for (int i = 0; i + 1 < NE; i += 2) evader_pair(i);
      if (NE & 1) evader_one(NE - 1);
    }
    __syncthreads();  // every sum is complete; the padded block is free
    const int next = o + gridDim.x;
    if (next < a.outer) stage_block(next);
    cp_async_commit();

    // C: the update, a thread per cell, kCBatch cells at a time (their
    // loads first)
    const float *base_o = s.base ? s.base + j0 : nullptr;
    for (int e0 = tid; e0 < inner; e0 += kCBatch * kColThreads) {
      float fv[kCBatch], bv[kCBatch], tv[kCBatch];
#pragma unroll
      for (int h = 0; h < kCBatch; h++) {
        const int c = min(e0 + h * kColThreads, inner - 1);
        fv[h] = __ldg(src_o + c);
        bv[h] = base_o ? __ldg(base_o + c) : fv[h];
        tv[h] = part[c];
      }
#pragma unroll
      for (int h = 0; h < kCBatch; h++) {
        const int c = e0 + h * kColThreads;
        if (c >= inner) break;
        const int64_t j = j0 + c;
        float value = fmaf(s.dt, tv[h], fv[h]);
        if (base_o) value = 0.5f * (bv[h] + value);
        if (g.order == 1 || base_o) {
          const float previous = bv[h];  // the partner, or the stage input
          const float tube = previous < value ? previous : value;
          value = tube < avoid ? avoid : tube;
          if (previous > 0.f && value <= 0.f && isnan(s.arrival[j]))
            s.arrival[j] = (float)s.tau + s.dt * previous / (previous - value);
          change_max = fmaxf(change_max, fabsf(value - previous));
        }
        bad |= !isfinite(value);
        s.dst[j] = value;
      }
    }
  }
  cp_async_wait_all();

  if (__syncthreads_or(bad) && tid == 0) atomicOr(&s.stats->nonfinite, 1u);
  for (int off = 16; off > 0; off >>= 1)
    change_max = fmaxf(change_max, __shfl_xor_sync(0xffffffffu, change_max, off));
  if (lane == 0) warp_max[warp] = change_max;
  __syncthreads();
  if (tid == 0) {
    float m = 0.f;
    for (int w = 0; w < nwarps; w++) m = fmaxf(m, warp_max[w]);
    if (m > 0.f)
      atomicMax(&s.stats->residual, (unsigned long long)__double_as_longlong((double)m));
  }
}

template <int ORDER, int NE, int SKIND>
cudaError_t launch_column_kind(const ColW8Args &a, size_t smem, cudaStream_t stream) {
  auto kernel = world8_column_kernel<ORDER, NE, SKIND>;
  static size_t configured = 0;
  static int resident = 0;
  if (configured != smem || resident == 0) {
    cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kColThreads, smem);
    if (e != cudaSuccess) return e;
    if (resident < 1) return cudaErrorInvalidConfiguration;
    configured = smem;
  }
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = a.outer < sms * resident ? a.outer : sms * resident;
  kernel<<<blocks, kColThreads, smem, stream>>>(a);
  return cudaGetLastError();
}

template <int ORDER, int NE>
cudaError_t launch_column_ne(const ColW8Args &a, size_t smem, cudaStream_t stream) {
  return a.g.linear_speed ? launch_column_kind<ORDER, NE, kInward>(a, smem, stream)
                          : launch_column_kind<ORDER, NE, kExtrapolated>(a, smem, stream);
}

template <int ORDER>
cudaError_t launch_column(const ColW8Args &a, size_t smem, cudaStream_t stream) {
  switch (a.g.shape[7]) {
    case 3: return launch_column_ne<ORDER, 3>(a, smem, stream);
    case 4: return launch_column_ne<ORDER, 4>(a, smem, stream);
    case 5: return launch_column_ne<ORDER, 5>(a, smem, stream);
    case 6: return launch_column_ne<ORDER, 6>(a, smem, stream);
    case 7: return launch_column_ne<ORDER, 7>(a, smem, stream);
    default: return launch_column_ne<ORDER, 8>(a, smem, stream);
  }
}
}  // namespace

cudaError_t world8_stage_fast(const World8Grid &g, const World8Stage &s,
                              cudaStream_t stream) {
  const int64_t inner = (int64_t)g.shape[4] * g.shape[5] * g.shape[6] * g.shape[7];
  // the column kernel: vE columns of 3 to 8 nodes, two CTAs per SM
  if (g.shape[7] >= 3 && g.shape[7] <= 8 && column_smem_bytes(g) <= kMaxColumnBytes) {
    ColW8Args c;
    c.g = g;
    c.s = s;
    c.inner = (int)inner;
    c.outer = (int)(g.cells / inner);
    c.ncols = (int)(inner / g.shape[7]);
    c.dnh = make_divisor(g.nh);
    c.dn = make_divisor(g.n);
    const size_t smem = column_smem_bytes(g);
    return g.order == 1 ? launch_column<1>(c, smem, stream) : launch_column<2>(c, smem, stream);
  }
  if (inner * 4 > kMaxBlockBytes) return w8::launch_stage<true>(g, s, stream);
  FastW8Args a;
  a.g = g;
  a.s = s;
  a.inner = (int)inner;
  a.outer = (int)(g.cells / inner);
  a.d7 = make_divisor(g.shape[7]);
  a.d6 = make_divisor(g.shape[6]);
  a.d5 = make_divisor(g.shape[5]);
  const size_t smem = (size_t)2 * inner * sizeof(float);
  return g.order == 1 ? launch_block<1>(a, smem, stream) : launch_block<2>(a, smem, stream);
}

}  // namespace pe
