// Relative 5D ENO/LF stage, fast variant: float32 storage and float32 local
// arithmetic, one launch per RK stage (native_relative.cpp:124-172).
//
// Work decomposition.  A CTA owns `rows` consecutive y rows of one (vP, vE)
// pair and sweeps `psi_chunk` consecutive headings.  A thread owns one
// 16-byte chunk of 4 consecutive x cells in one row.  For each heading step
// the CTA needs, in shared memory:
//   * its own (vP, vE) plane at headings psi-2 .. psi+2, rows y0-2 .. y0+R+1
//     (the heading window and the y halo), kept in a ring of 6 slots;
//   * the 8 neighbour planes (vE+-1, vE+-2, vP+-1, vP+-2) at the current
//     heading, rows y0 .. y0+R-1, in a ring of 2 slots.
// All of it arrives by bulk asynchronous copies (the TMA engine,
// cp.async.bulk) that complete on mbarriers; thread 0 issues the copies two
// heading steps ahead, so the 4-cell chunks are computed from shared memory
// while the next planes stream in.  Every wait is bounded: a wait that gives
// up sets the handle's timeout flag instead of hanging.
//
// Arithmetic.  The 4 cells of a chunk are processed as two float2 pairs with
// sm_100 packed FP32 instructions (__ffma2_rn / __fadd2_rn / __fmul2_rn).
// Second differences are kept unscaled (h^2 * D2) and the ENO2 slope is
// (first difference +- 0.5 * selected second difference) / h -- the
// reference's dm + 0.5*h*D2 rewritten.  Along x the edge differences and the
// ENO selection between neighbouring cells of a chunk are shared.  Results
// agree with the double-local reference to float rounding except where an
// ENO selection is tied to rounding; relative5d_exact.cu is the bit-exact
// path.
#include <cstdio>

#include "relative5d.cuh"

namespace pe {
namespace {

constexpr int OWN_SLOTS = 6;
constexpr int NB_SLOTS = 2;
constexpr int NEIGHBOURS = 8;  // vE-2, vE-1, vE+1, vE+2, vP-2, vP-1, vP+1, vP+2
constexpr int MAX_THREADS = 512;
constexpr unsigned WAIT_LIMIT = 1u << 22;

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile(
      "{\n .reg .b64 state;\n"
      " mbarrier.arrive.expect_tx.shared::cta.b64 state, [%0], %1;\n}" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bulk copy global -> shared (16-byte aligned, size multiple of 16) that
// signals `bar` with its byte count.
__device__ __forceinline__ void bulk_load(void *dst, const void *src,
                                          uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for one mbarrier phase.  Returns false (and flags the handle)
// when the limit is reached.
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t parity,
                                           unsigned int *timeout_flag) {
  for (unsigned i = 0; i < WAIT_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(timeout_flag, 1u);
  return false;
}

// ------------------------------------------------------------ float2 helpers
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {  // a - b
  return __ffma2_rn(b, f2(-1.f), a);
}
__device__ __forceinline__ float eno_pick(float a, float b) {
  return fabsf(a) < fabsf(b) ? a : b;
}
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// Backward/forward ENO slopes (unscaled by 1/h) of a pair of cells along a
// non-x axis from their five values.  GENERAL handles the end nodes of a
// non-periodic axis (pos is the same for both cells of the pair).
template <int ORDER, bool GENERAL>
__device__ __forceinline__ void slope_pair(float2 m2, float2 m1, float2 v,
                                           float2 p1, float2 p2, int pos,
                                           int n, float2 &lo, float2 &hi) {
  const float2 d_lo = sub2(v, m1), d_hi = sub2(p1, v);
  if (ORDER == 1) {
    lo = d_lo;
    hi = d_hi;
  } else {
    const float2 c2 = sub2(d_hi, d_lo);
    float2 l2 = sub2(d_lo, sub2(m1, m2));
    float2 r2 = sub2(sub2(p2, p1), d_hi);
    if (GENERAL) {
      if (pos < 2) l2 = c2;
      if (pos + 2 >= n) r2 = c2;
    }
    const float2 pick_lo = make_float2(eno_pick(l2.x, c2.x), eno_pick(l2.y, c2.y));
    const float2 pick_hi = make_float2(eno_pick(c2.x, r2.x), eno_pick(c2.y, r2.y));
    lo = __ffma2_rn(f2(0.5f), pick_lo, d_lo);
    hi = __ffma2_rn(f2(-0.5f), pick_hi, d_hi);
  }
  if (GENERAL) {
    if (pos == 0) lo = hi = d_hi;
    if (pos == n - 1) lo = hi = d_lo;
  }
}

template <int ORDER>
__device__ __forceinline__ void slope_pair_any(float2 m2, float2 m1, float2 v,
                                               float2 p1, float2 p2, int pos,
                                               int n, float2 &lo, float2 &hi) {
  if (pos >= 2 && pos + 2 < n)
    slope_pair<ORDER, false>(m2, m1, v, p1, p2, pos, n, lo, hi);
  else
    slope_pair<ORDER, true>(m2, m1, v, p1, p2, pos, n, lo, hi);
}

// ENO slopes along x for the 4 cells x0..x0+3 from the window x0-2..x0+5,
// sharing edge differences and ENO selections between neighbouring cells.
template <int ORDER>
__device__ __forceinline__ void slopes_x(const float w[8], int x0, int nx,
                                         float lo[4], float hi[4]) {
  float e[7];
#pragma unroll
  for (int i = 0; i < 7; i++) e[i] = w[i + 1] - w[i];
  if (ORDER == 1) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = e[i + 1];
      hi[i] = e[i + 2];
    }
  } else {
    float d2[7];
#pragma unroll
    for (int k = 1; k < 7; k++) d2[k] = e[k] - e[k - 1];
    float m[7];  // m[k], k = 2..6: selection between nodes k-1 and k
#pragma unroll
    for (int k = 2; k < 7; k++) m[k] = eno_pick(d2[k - 1], d2[k]);
    // Next to an end the missing outer second difference is replaced by the
    // centred one (native_relative.cpp:58-63).
    if (x0 == 0) m[3] = d2[3];
    const int k_end = nx - x0;  // window node of x = nx-2
    if (k_end >= 2 && k_end <= 5) {
#pragma unroll
      for (int k = 2; k <= 5; k++)
        if (k == k_end) m[k + 1] = d2[k];
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = fmaf(0.5f, m[i + 2], e[i + 1]);
      hi[i] = fmaf(-0.5f, m[i + 3], e[i + 2]);
    }
  }
  // One-sided first differences at the two end nodes.
  if (x0 == 0) lo[0] = hi[0] = e[2];
  const int i_end = nx - 1 - x0;
  if (i_end >= 0 && i_end < 4) {
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (i == i_end) lo[i] = hi[i] = e[i + 1];
  }
}

struct FastArgs {
  Rel5Grid g;
  Rel5Stage s;
  int rows, psi_chunk, slabs, chunks, xc;
  float ihx, ihp, ihv, ihe;
  float dt;
};

template <int ORDER, int BLEND>
__global__ void __launch_bounds__(MAX_THREADS)
    rel5_stage_tma_kernel(const FastArgs a) {
  extern __shared__ __align__(128) float smem[];
  const Rel5Grid &g = a.g;
  const int R = a.rows, XP = g.xp;
  const int own_floats = (R + 4) * XP;
  const int nb_floats = R * XP;
  float *own = smem;                                      // [6][R+4][XP]
  float *nbr = own + OWN_SLOTS * own_floats;              // [2][8][R][XP]
  uint64_t *bars = reinterpret_cast<uint64_t *>(nbr + NB_SLOTS * NEIGHBOURS * nb_floats);
  uint64_t *own_bar = bars, *nb_bar = bars + OWN_SLOTS;
  float *red = reinterpret_cast<float *>(bars + OWN_SLOTS + NB_SLOTS);

  // Block -> (slab, vE, vP, heading chunk); the heading chunk is outermost so
  // that resident CTAs share the planes of a few headings in L2.
  int b = blockIdx.x;
  const int slab = b % a.slabs;
  b /= a.slabs;
  const int ie = b % g.nve;
  b /= g.nve;
  const int iv = b % g.nvp;
  const int chunk = b / g.nvp;
  const int y0 = slab * R;
  const int r_eff = min(R, g.nx - y0);
  const int p0 = chunk * a.psi_chunk;
  const int steps = min(a.psi_chunk, g.nh - p0);
  const int64_t PP = (int64_t)g.nx * XP;  // plane pitch

  const int tid = threadIdx.x;
  const int r = tid / a.xc, c = tid % a.xc;
  const bool active = r < r_eff;
  const int x0 = 4 * c;

  // Neighbour planes that exist (uniform per CTA).
  const int nb_e[NEIGHBOURS] = {ie - 2, ie - 1, ie + 1, ie + 2, ie, ie, ie, ie};
  const int nb_v[NEIGHBOURS] = {iv, iv, iv, iv, iv - 2, iv - 1, iv + 1, iv + 2};

  // Copies are issued by thread 0 only.
  const int row_lo = max(0, y0 - 2), row_hi = min(g.nx, y0 + r_eff + 2);
  auto plane_index = [&](int v_idx, int e_idx, int psi) -> int64_t {
    return ((int64_t)v_idx * g.nve + e_idx) * g.nh + psi;
  };
  auto issue_own = [&](int d) {  // own plane at relative heading d
    const int slot = (d + 2) % OWN_SLOTS;
    const int psi = ((p0 + d) % g.nh + g.nh) % g.nh;
    const float *src = a.s.src + plane_index(iv, ie, psi) * PP + (int64_t)row_lo * XP;
    float *dst = own + slot * own_floats + (row_lo - (y0 - 2)) * XP;
    const uint32_t bytes = (uint32_t)((row_hi - row_lo) * XP * 4);
    mbar_expect_tx(&own_bar[slot], bytes);
    bulk_load(dst, src, bytes, &own_bar[slot]);
  };
  auto issue_nb = [&](int k) {  // neighbour planes for step k
    const int slot = k % NB_SLOTS;
    const int psi = p0 + k;
    uint32_t total = 0;
    const uint32_t bytes = (uint32_t)(r_eff * XP * 4);
#pragma unroll
    for (int q = 0; q < NEIGHBOURS; q++)
      if (nb_e[q] >= 0 && nb_e[q] < g.nve && nb_v[q] >= 0 && nb_v[q] < g.nvp)
        total += bytes;
    mbar_expect_tx(&nb_bar[slot], total);
#pragma unroll
    for (int q = 0; q < NEIGHBOURS; q++)
      if (nb_e[q] >= 0 && nb_e[q] < g.nve && nb_v[q] >= 0 && nb_v[q] < g.nvp)
        bulk_load(nbr + (slot * NEIGHBOURS + q) * nb_floats,
                  a.s.src + plane_index(nb_v[q], nb_e[q], psi) * PP + (int64_t)y0 * XP,
                  bytes, &nb_bar[slot]);
  };

  if (tid == 0) {
    for (int i = 0; i < OWN_SLOTS + NB_SLOTS; i++) mbar_init(&bars[i], 1);
    fence_barrier_init();
  }
  // Rows of the y halo outside the grid are never copied: zero them once.
  for (int slot = 0; slot < OWN_SLOTS; slot++)
    for (int i = tid; i < (R + 4) * XP; i += blockDim.x) {
      const int row = y0 - 2 + i / XP;
      if (row < 0 || row >= g.nx) own[slot * own_floats + i] = 0.f;
    }
  __syncthreads();
  int last_own = -3, last_nb = -1;  // latest issued (thread 0)
  if (tid == 0) {
    for (int d = -2; d <= 3 && d <= steps + 1; d++) {
      issue_own(d);
      last_own = d;
    }
    for (int k = 0; k < NB_SLOTS && k < steps; k++) {
      issue_nb(k);
      last_nb = k;
    }
  }

  // Per-thread constants.
  const float ext = (float)g.extent, dxf = (float)g.dx;
  const float vp = (float)(g.vp_lo + iv * g.dvp);
  const float ve = (float)(g.ve_lo + ie * g.dve);
  const float wp = fabsf(vp) * (float)g.curv_p;
  const float we = fabsf(ve) * (float)g.curv_e;
  const float ap = (float)g.acc_p, ae = (float)g.acc_e;
  const float plo = iv == 0 ? 0.f : -ap, phi = iv == g.nvp - 1 ? 0.f : ap;
  const float elo = ie == 0 ? 0.f : -ae, ehi = ie == g.nve - 1 ? 0.f : ae;
  const bool p_inner = iv > 0 && iv < g.nvp - 1;
  const bool e_inner = ie > 0 && ie < g.nve - 1;
  const int iy = y0 + r;
  const float y = fmaf((float)iy, dxf, -ext);
  float xs[4];
#pragma unroll
  for (int i = 0; i < 4; i++) xs[i] = fmaf((float)(x0 + i), dxf, -ext);
  const float2 negx_a = make_float2(-xs[0], -xs[1]), negx_b = make_float2(-xs[2], -xs[3]);
  const float2 absx_a = make_float2(fabsf(xs[0]), fabsf(xs[1]));
  const float2 absx_b = make_float2(fabsf(xs[2]), fabsf(xs[3]));
  const float hx = 0.5f * a.ihx, hp = 0.5f * a.ihp, hv = 0.5f * a.ihv, he = 0.5f * a.ihe;
  const float dt = a.dt;
  const int ctr = (r + 2) * XP + x0;  // this chunk in an own slot

  float residual = 0.f;
  float2 finite_acc = f2(0.f);
  bool alive = true;
  unsigned int *timeout = &a.s.stats->timeout;

  for (int k = 0; k < steps; k++) {
    // Wait for own planes up to k+2 and the neighbour planes of step k.
    if (alive) {
      for (int d = (k == 0 ? -2 : k + 2); d <= k + 2 && d <= steps + 1; d++)
        alive &= wait_phase(&own_bar[(d + 2) % OWN_SLOTS], ((d + 2) / OWN_SLOTS) & 1, timeout);
      if (alive) alive &= wait_phase(&nb_bar[k % NB_SLOTS], (k / NB_SLOTS) & 1, timeout);
    }
    const int ip = p0 + k;
    if (active && alive) {
      const float *o0 = own + ((k + 2) % OWN_SLOTS) * own_floats;  // heading k
      const float *om1 = own + ((k + 1) % OWN_SLOTS) * own_floats;
      const float *om2 = own + ((k) % OWN_SLOTS) * own_floats;
      const float *op1 = own + ((k + 3) % OWN_SLOTS) * own_floats;
      const float *op2 = own + ((k + 4) % OWN_SLOTS) * own_floats;
      const float *nb = nbr + (k % NB_SLOTS) * NEIGHBOURS * nb_floats + r * XP + x0;

      const float4 C = *reinterpret_cast<const float4 *>(o0 + ctr);
      const float2 v_a = lo2(C), v_b = hi2(C);

      // x: window x0-2 .. x0+5
      const float2 xl = *reinterpret_cast<const float2 *>(o0 + ctr - 2);
      const float2 xr = *reinterpret_cast<const float2 *>(o0 + ctr + 4);
      const float w[8] = {xl.x, xl.y, C.x, C.y, C.z, C.w, xr.x, xr.y};
      float xlo[4], xhi[4];
      slopes_x<ORDER>(w, x0, g.nx, xlo, xhi);
      const float2 lx_a = make_float2(xlo[0], xlo[1]), lx_b = make_float2(xlo[2], xlo[3]);
      const float2 hx_a = make_float2(xhi[0], xhi[1]), hx_b = make_float2(xhi[2], xhi[3]);

      // y: rows iy-2 .. iy+2 of heading k
      float2 ly_a, ly_b, hy_a, hy_b;
      {
        const float4 m2 = *reinterpret_cast<const float4 *>(o0 + ctr - 2 * XP);
        const float4 m1 = *reinterpret_cast<const float4 *>(o0 + ctr - XP);
        const float4 p1 = *reinterpret_cast<const float4 *>(o0 + ctr + XP);
        const float4 p2 = *reinterpret_cast<const float4 *>(o0 + ctr + 2 * XP);
        slope_pair_any<ORDER>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), iy, g.nx, ly_a, hy_a);
        slope_pair_any<ORDER>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), iy, g.nx, ly_b, hy_b);
      }
      // psi: periodic, the ring holds headings k-2 .. k+2
      float2 lp_a, lp_b, hp_a, hp_b;
      {
        const float4 m2 = *reinterpret_cast<const float4 *>(om2 + ctr);
        const float4 m1 = *reinterpret_cast<const float4 *>(om1 + ctr);
        const float4 p1 = *reinterpret_cast<const float4 *>(op1 + ctr);
        const float4 p2 = *reinterpret_cast<const float4 *>(op2 + ctr);
        slope_pair<ORDER, false>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), 2, 5, lp_a, hp_a);
        slope_pair<ORDER, false>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), 2, 5, lp_b, hp_b);
      }
      // vE and vP: neighbour slots
      float2 le_a, le_b, he_a, he_b, lv_a, lv_b, hv_a, hv_b;
      {
        const float4 m2 = *reinterpret_cast<const float4 *>(nb + 0 * nb_floats);
        const float4 m1 = *reinterpret_cast<const float4 *>(nb + 1 * nb_floats);
        const float4 p1 = *reinterpret_cast<const float4 *>(nb + 2 * nb_floats);
        const float4 p2 = *reinterpret_cast<const float4 *>(nb + 3 * nb_floats);
        slope_pair_any<ORDER>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), ie, g.nve, le_a, he_a);
        slope_pair_any<ORDER>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), ie, g.nve, le_b, he_b);
      }
      {
        const float4 m2 = *reinterpret_cast<const float4 *>(nb + 4 * nb_floats);
        const float4 m1 = *reinterpret_cast<const float4 *>(nb + 5 * nb_floats);
        const float4 p1 = *reinterpret_cast<const float4 *>(nb + 6 * nb_floats);
        const float4 p2 = *reinterpret_cast<const float4 *>(nb + 7 * nb_floats);
        slope_pair_any<ORDER>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), iv, g.nvp, lv_a, hv_a);
        slope_pair_any<ORDER>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), iv, g.nvp, lv_b, hv_b);
      }

      // Hamiltonian + dissipation (native_relative.cpp:144-157).
      const float bx = fmaf(ve, __ldg(a.s.csf + ip), -vp);
      const float by = ve * __ldg(a.s.snf + ip);
      const float2 bx2 = f2(bx), by2 = f2(by);
      const float ax_coef = fmaf(wp, fabsf(y), fabsf(bx)) * a.ihx;  // alpha_x / h
      const float ap_coef = (wp + we) * a.ihp, av_coef = ap * a.ihv, ae_coef = ae * a.ihe;
      const float2 absby = f2(fabsf(by));
      const float4 prev4 =
          BLEND ? *reinterpret_cast<const float4 *>(
                      a.s.dst + plane_index(iv, ie, ip) * PP + (int64_t)iy * XP + x0)
                : C;

      float2 out[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const float2 lx = h ? lx_b : lx_a, hxv = h ? hx_b : hx_a;
        const float2 ly = h ? ly_b : ly_a, hy = h ? hy_b : hy_a;
        const float2 lp = h ? lp_b : lp_a, hpv = h ? hp_b : hp_a;
        const float2 lv = h ? lv_b : lv_a, hvv = h ? hv_b : hv_a;
        const float2 le = h ? le_b : le_a, hev = h ? he_b : he_a;
        const float2 v = h ? v_b : v_a;
        const float2 negx = h ? negx_b : negx_a, absx = h ? absx_b : absx_a;
        // centred gradients g = (lo + hi) / (2h); jumps hi - lo (unscaled)
        const float2 gx = __fmul2_rn(__fadd2_rn(lx, hxv), f2(hx));
        const float2 gy = __fmul2_rn(__fadd2_rn(ly, hy), f2(hx));
        const float2 gpn = __fmul2_rn(__fadd2_rn(lp, hpv), f2(-hp));  // -gp
        const float2 gv = __fmul2_rn(__fadd2_rn(lv, hvv), f2(hv));
        const float2 ge = __fmul2_rn(__fadd2_rn(le, hev), f2(he));
        float2 H = __ffma2_rn(by2, gy, __fmul2_rn(bx2, gx));
        float2 t = __ffma2_rn(f2(y), gx, gpn);  // y*gx - gp
        t = __ffma2_rn(negx, gy, t);             // - x*gy
        float hs[2] = {H.x, H.y};
        const float ts[2] = {t.x, t.y}, gps[2] = {gpn.x, gpn.y};
        const float gvs[2] = {gv.x, gv.y}, ges[2] = {ge.x, ge.y};
#pragma unroll
        for (int l = 0; l < 2; l++) {
          hs[l] = fmaf(-wp, fabsf(ts[l]), hs[l]);
          hs[l] = fmaf(we, fabsf(gps[l]), hs[l]);
          hs[l] += p_inner ? -ap * fabsf(gvs[l]) : fminf(plo * gvs[l], phi * gvs[l]);
          hs[l] += e_inner ? ae * fabsf(ges[l]) : fmaxf(elo * ges[l], ehi * ges[l]);
        }
        H = make_float2(hs[0], hs[1]);
        // dissipation: sum alpha_k/h_k * (hi - lo)_k
        const float2 ay = __fmul2_rn(__ffma2_rn(f2(wp), absx, absby), f2(a.ihx));
        float2 diss = __fmul2_rn(f2(ax_coef), sub2(hxv, lx));
        diss = __ffma2_rn(ay, sub2(hy, ly), diss);
        diss = __ffma2_rn(f2(ap_coef), sub2(hpv, lp), diss);
        diss = __ffma2_rn(f2(av_coef), sub2(hvv, lv), diss);
        diss = __ffma2_rn(f2(ae_coef), sub2(hev, le), diss);
        H = __ffma2_rn(f2(0.5f), diss, H);
        float2 value = __ffma2_rn(f2(dt), make_float2(fminf(H.x, 0.f), fminf(H.y, 0.f)), v);
        const float2 prev = BLEND ? (h ? hi2(prev4) : lo2(prev4)) : v;
        if (BLEND) value = __fmul2_rn(f2(0.5f), __fadd2_rn(prev, value));
        if (x0 + 2 * h + 1 >= g.nx) {  // row padding stays 0
          if (x0 + 2 * h >= g.nx) value.x = 0.f;
          value.y = 0.f;
        }
        finite_acc = __ffma2_rn(value, f2(0.f), finite_acc);
        out[h] = value;
        if (BLEND || ORDER == 1) {
          const float2 change = sub2(value, prev);
          residual = fmaxf(residual, fmaxf(fabsf(change.x), fabsf(change.y)));
          const float pv[2] = {prev.x, prev.y}, nv[2] = {value.x, value.y};
#pragma unroll
          for (int l = 0; l < 2; l++) {
            const int ix = x0 + 2 * h + l;
            if (pv[l] > 0.f && nv[l] <= 0.f && ix < g.nx) {
              float *slot = a.s.arrival + plane_index(iv, ie, ip) * PP +
                            (int64_t)iy * XP + ix;
              if (isnan(*slot))
                *slot = (float)(a.s.t + a.s.dt * (double)pv[l] /
                                            ((double)pv[l] - (double)nv[l]));
            }
          }
        }
      }
      const float4 result = make_float4(out[0].x, out[0].y, out[1].x, out[1].y);
      *reinterpret_cast<float4 *>(a.s.dst + plane_index(iv, ie, ip) * PP +
                                  (int64_t)iy * XP + x0) = result;
    }
    __syncthreads();
    // Refill: the slot of heading k-2 and the neighbour slot of step k are
    // free now.
    if (tid == 0 && alive) {
      fence_async_shared();
      if (k + 4 <= steps + 1) {
        issue_own(k + 4);
        last_own = k + 4;
      }
      if (k + 2 < steps) {
        issue_nb(k + 2);
        last_nb = k + 2;
      }
    }
  }

  // Block reductions: non-finite flag and the largest change.
  const bool bad = active && !(isfinite(finite_acc.x) && isfinite(finite_acc.y));
  if (__syncthreads_or(bad) && tid == 0) atomicOr(&a.s.stats->nonfinite, 1u);
  if (BLEND || ORDER == 1) {
    for (int off = 16; off > 0; off >>= 1)
      residual = fmaxf(residual, __shfl_xor_sync(0xffffffffu, residual, off));
    if ((tid & 31) == 0) red[tid >> 5] = residual;
    __syncthreads();
    if (tid == 0) {
      float m = 0.f;
      for (int w = 0; w < (int)((blockDim.x + 31) >> 5); w++) m = fmaxf(m, red[w]);
      if (m > 0.f)
        atomicMax(&a.s.stats->residual,
                  (unsigned long long)__double_as_longlong((double)m));
    }
  }
  if (__syncthreads_or(!alive) && tid == 0) {
    // A wait gave up: wait (bounded) for the last phase issued on every
    // barrier, so no copy is still writing this CTA's shared memory when it
    // exits.  Phases complete in order.
    for (int d = last_own; d >= last_own - OWN_SLOTS + 1 && d >= -2; d--)
      for (unsigned i = 0; i < WAIT_LIMIT; i++)
        if (mbar_try_wait(&own_bar[(d + 2) % OWN_SLOTS], ((d + 2) / OWN_SLOTS) & 1)) break;
    for (int k = last_nb; k >= last_nb - NB_SLOTS + 1 && k >= 0; k--)
      for (unsigned i = 0; i < WAIT_LIMIT; i++)
        if (mbar_try_wait(&nb_bar[k % NB_SLOTS], (k / NB_SLOTS) & 1)) break;
  }
}

template <int ORDER, int BLEND>
cudaError_t launch(const FastArgs &args, size_t smem, int threads, int blocks,
                   cudaStream_t stream) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(rel5_stage_tma_kernel<ORDER, BLEND>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         227 * 1024);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  rel5_stage_tma_kernel<ORDER, BLEND><<<blocks, threads, smem, stream>>>(args);
  return cudaGetLastError();
}

__global__ void rel5_init_kernel(const float *__restrict__ plane,
                                 float *__restrict__ field,
                                 float *__restrict__ arrival, int64_t n_padded,
                                 int nx, int xp, float start_time) {
  const int64_t pp = (int64_t)nx * xp;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n_padded;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t in_plane = j % pp;
    const int ix = (int)(in_plane % xp);
    const int iy = (int)(in_plane / xp);
    if (ix >= nx) {
      field[j] = 0.f;
      arrival[j] = 0.f;
      continue;
    }
    const float v = plane ? plane[iy * nx + ix] : field[j];
    if (plane) field[j] = v;
    arrival[j] = v <= 0.f ? start_time : __int_as_float(0x7fc00000);
  }
}

// Dense [.., y, x] <-> padded [.., y, xp] row conversion.
__global__ void rel5_pack_kernel(const float *__restrict__ padded,
                                 float *__restrict__ dense, int64_t rows, int nx,
                                 int xp) {
  const int64_t n = rows * nx;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    dense[j] = padded[(j / nx) * xp + j % nx];
}

__global__ void rel5_unpack_kernel(const float *__restrict__ dense,
                                   float *__restrict__ padded, int64_t rows,
                                   int nx, int xp) {
  const int64_t n = rows * xp;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(j % xp);
    padded[j] = ix < nx ? dense[(j / xp) * nx + ix] : 0.f;
  }
}

}  // namespace

cudaError_t rel5_pack(const Rel5Grid &g, const float *padded, float *dense,
                      cudaStream_t stream) {
  const int64_t rows = g.n / g.nx;
  rel5_pack_kernel<<<148 * 16, 256, 0, stream>>>(padded, dense, rows, g.nx, g.xp);
  return cudaGetLastError();
}

cudaError_t rel5_unpack(const Rel5Grid &g, const float *dense, float *padded,
                        cudaStream_t stream) {
  const int64_t rows = g.n / g.nx;
  rel5_unpack_kernel<<<148 * 16, 256, 0, stream>>>(dense, padded, rows, g.nx, g.xp);
  return cudaGetLastError();
}

size_t rel5_fast_smem_bytes(const Rel5Grid &g, const Rel5Tile &t) {
  const size_t own = (size_t)OWN_SLOTS * (t.rows + 4) * g.xp;
  const size_t nb = (size_t)NB_SLOTS * NEIGHBOURS * t.rows * g.xp;
  return 4 * (own + nb) + 8 * (OWN_SLOTS + NB_SLOTS) + 4 * (MAX_THREADS / 32);
}

Rel5Tile rel5_default_tile(const Rel5Grid &g) {
  const int xc = g.xp / 4;
  Rel5Tile t{1, 12};
  // rows: at most 256 threads, fewest idle rows, then most rows.
  int best_waste = 1 << 30;
  for (int rows = 1; rows * xc <= 256 && rows <= g.nx; rows++) {
    const int slabs = (g.nx + rows - 1) / rows;
    const int waste = slabs * rows - g.nx;
    if (waste < best_waste || (waste == best_waste && rows > t.rows)) {
      best_waste = waste;
      t.rows = rows;
    }
  }
  t.psi_chunk = g.nh < 12 ? g.nh : 12;
  return t;
}

cudaError_t rel5_stage_f32(const Rel5Grid &g, const Rel5Tile &t,
                           const Rel5Stage &s, int blend, cudaStream_t stream) {
  FastArgs args;
  args.g = g;
  args.s = s;
  args.rows = t.rows;
  args.psi_chunk = t.psi_chunk;
  args.xc = g.xp / 4;
  args.slabs = (g.nx + t.rows - 1) / t.rows;
  args.chunks = (g.nh + t.psi_chunk - 1) / t.psi_chunk;
  args.ihx = (float)(1.0 / g.dx);
  args.ihp = (float)(1.0 / g.dphi);
  args.ihv = (float)(1.0 / g.dvp);
  args.ihe = (float)(1.0 / g.dve);
  args.dt = (float)s.dt;
  const int threads = ((t.rows * args.xc + 31) / 32) * 32;
  if (threads > MAX_THREADS) return cudaErrorInvalidConfiguration;
  const size_t smem = rel5_fast_smem_bytes(g, t);
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  const int blocks = args.slabs * g.nve * g.nvp * args.chunks;
  if (g.order == 1) return launch<1, 0>(args, smem, threads, blocks, stream);
  if (blend) return launch<2, 1>(args, smem, threads, blocks, stream);
  return launch<2, 0>(args, smem, threads, blocks, stream);
}

cudaError_t rel5_init(const Rel5Grid &g, const float *plane, float *field,
                      float *arrival, float start_time, cudaStream_t stream) {
  const int threads = 256;
  int64_t blocks = (g.n_padded + threads - 1) / threads;
  if (blocks > 148 * 64) blocks = 148 * 64;
  rel5_init_kernel<<<(unsigned)blocks, threads, 0, stream>>>(
      plane, field, arrival, g.n_padded, g.nx, g.xp, start_time);
  return cudaGetLastError();
}

}  // namespace pe
