// Relative 5D ENO/LF stage, fast variant: float32 storage and float32 local
// arithmetic, one launch per RK stage (native_relative.cpp:124-172).
//
// Work decomposition.  A work item is `rows` consecutive y rows of one
// (vP, vE) pair over `psi_chunk` consecutive headings; a persistent CTA walks
// a strided list of items.  A thread owns one 16-byte chunk of 4 consecutive
// x cells in one row.  For each heading step the CTA needs, in shared memory:
//   * its own (vP, vE) plane, rows y0-2 .. y0+R+1 (the y halo), in a ring of
//     6 slots: the current heading for the y and x neighbours and the heading
//     two ahead to refill each thread's 5-heading register window;
//   * the 8 neighbour planes (vE+-1, vE+-2, vP+-1, vP+-2) at the current
//     heading, rows y0 .. y0+R-1, in a ring of 2 slots.
// All of it arrives by bulk asynchronous copies (the TMA engine,
// cp.async.bulk) issued by a producer warp that runs ahead across items, and
// completes on mbarriers.  Every wait is bounded: a wait that gives up sets
// the handle's timeout flag instead of hanging.
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
#include <algorithm>
#include <cstdio>

#include "relative5d.cuh"
#include "relative5d_eno_f32.cuh"

namespace pe {
namespace {

using namespace eno32;

constexpr int OWN_SLOTS = 6;
constexpr int NB_SLOTS = 2;
constexpr int NEIGHBOURS = 8;  // vE-2, vE-1, vE+1, vE+2, vP-2, vP-1, vP+1, vP+2
// a neighbour set also holds, on RK2 stage 2, the item's rows of the
// stage's old value V (the blend partner), prefetched with the neighbours
constexpr int NB_PLANES = NEIGHBOURS + 1;
constexpr int MAX_THREADS = 512;
constexpr int TARGET_THREADS = 256;  // launch bound: two CTAs of 256 per SM
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

struct FastArgs {
  Rel5Grid g;
  Rel5Stage s;
  int rows, psi_chunk, slabs, chunks, xc, consumer_warps, items;
  int vp_first, vp_count;  // the vP slabs this launch updates (a shard's own)
  float ihx, ihp, ihv, ihe;
  float dt;
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile(
      "{\n .reg .b64 state;\n"
      " mbarrier.arrive.shared::cta.b64 state, [%0];\n}" ::"r"(smem_u32(bar))
      : "memory");
}

// Shared memory layout of one CTA.
struct SmemLayout {
  int own_floats, nb_floats;
  int own_off, nb_off;                 // floats
  int bar_off, red_off, trig_off;      // bytes
  int bytes;
};

__host__ __device__ inline SmemLayout smem_layout(int rows, int xp, int headings) {
  SmemLayout L;
  L.own_floats = (rows + 4) * xp;
  L.nb_floats = rows * xp;
  L.own_off = 0;
  L.nb_off = OWN_SLOTS * L.own_floats;
  L.bar_off = 4 * (L.nb_off + NB_SLOTS * NB_PLANES * L.nb_floats);
  L.red_off = L.bar_off + 8 * 2 * (OWN_SLOTS + NB_SLOTS);
  L.trig_off = L.red_off + 4 * (MAX_THREADS / 32);
  L.bytes = L.trig_off + 4 * 2 * headings;
  return L;
}

// One work item: `rows` y rows (from y0) of one (vP, vE) pair over `steps`
// headings from p0.  Items are numbered heading chunk first, so that the
// CTAs resident at any moment share the planes of a few headings in L2.
struct Item {
  int iv, ie, y0, r_eff, p0, steps;
};

__device__ __forceinline__ Item decode_item(const FastArgs &a, int idx) {
  Item it;
  const int slab = idx % a.slabs;
  idx /= a.slabs;
  it.ie = idx % a.g.nve;
  idx /= a.g.nve;
  it.iv = a.vp_first + idx % a.vp_count;
  const int chunk = idx / a.vp_count;
  it.y0 = slab * a.rows;
  it.r_eff = min(a.rows, a.g.nx - it.y0);
  it.p0 = chunk * a.psi_chunk;
  it.steps = min(a.psi_chunk, a.g.nh - it.p0);
  return it;
}

// Persistent, warp-specialised stage kernel.  Each CTA walks the items
// blockIdx.x, blockIdx.x + gridDim.x, ...  Warps 0..consumer_warps-1 compute
// 4-cell chunks; the last warp is the producer: its lane 0 issues every bulk
// copy in the order the consumers need them, across item boundaries, waiting
// on a ring slot's "empty" barrier (one arrival per consumer warp) before
// refilling it.  Consumers wait on the slots' "full" barriers.  Own planes of
// an item are numbered d = -2 .. steps+1; plane d is read at step d-2 (the
// heading window refill) and at step d (centre, y and x neighbours).
template <int ORDER, int BLEND>
__global__ void __launch_bounds__(TARGET_THREADS, 2)
    rel5_stage_kernel(const FastArgs a) {
  extern __shared__ __align__(128) float smem[];
  const Rel5Grid &g = a.g;
  const int R = a.rows, XP = g.xp;
  const SmemLayout L = smem_layout(R, XP, g.nh);
  float *own = smem + L.own_off;  // [6][R+4][XP]
  float *nbr = smem + L.nb_off;   // [2][8][R][XP]
  char *raw = reinterpret_cast<char *>(smem);
  uint64_t *bars = reinterpret_cast<uint64_t *>(raw + L.bar_off);
  uint64_t *own_full = bars, *own_empty = bars + OWN_SLOTS;
  uint64_t *nb_full = bars + 2 * OWN_SLOTS, *nb_empty = nb_full + NB_SLOTS;
  float *red = reinterpret_cast<float *>(raw + L.red_off);
  float *trig = reinterpret_cast<float *>(raw + L.trig_off);  // [nh][cos, sin]

  const int64_t PP = (int64_t)g.nx * XP;  // plane pitch
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool producer = warp == a.consumer_warps;
  unsigned int *timeout = &a.s.stats->timeout;
  auto plane_index = [&](int v_idx, int e_idx, int psi) -> int64_t {
    return ((int64_t)(v_idx - g.slab_lo) * g.nve + e_idx) * g.nh + psi;
  };

  if (tid == 0) {
    for (int i = 0; i < OWN_SLOTS; i++) {
      mbar_init(&own_full[i], 1);
      mbar_init(&own_empty[i], a.consumer_warps);
    }
    for (int i = 0; i < NB_SLOTS; i++) {
      mbar_init(&nb_full[i], 1);
      mbar_init(&nb_empty[i], a.consumer_warps);
    }
    fence_barrier_init();
  }
  for (int k = tid; k < g.nh; k += blockDim.x) {
    trig[2 * k] = __ldg(a.s.csf + k);
    trig[2 * k + 1] = __ldg(a.s.snf + k);
  }
  __syncthreads();

  float residual = 0.f;
  bool bad = false;
  bool alive = true;

  if (producer) {
    if (lane == 0) {
      unsigned og = 0, ng = 0;  // own planes / neighbour sets issued so far
      for (int idx = blockIdx.x; idx < a.items && alive; idx += gridDim.x) {
        const Item it = decode_item(a, idx);
        const int row_lo = max(0, it.y0 - 2), row_hi = min(g.nx, it.y0 + it.r_eff + 2);
        const uint32_t own_bytes = (uint32_t)((row_hi - row_lo) * XP * 4);
        const float *own_src = a.s.src + (int64_t)row_lo * XP;
        const int own_dst = (row_lo - (it.y0 - 2)) * XP;
        const uint32_t nb_bytes = (uint32_t)(it.r_eff * XP * 4);
        int nb_e[NEIGHBOURS], nb_v[NEIGHBOURS], nb_count = 0;
        {
          const int de[NEIGHBOURS] = {-2, -1, 1, 2, 0, 0, 0, 0};
          const int dv[NEIGHBOURS] = {0, 0, 0, 0, -2, -1, 1, 2};
          for (int q = 0; q < NEIGHBOURS; q++) {
            nb_e[q] = it.ie + de[q];
            nb_v[q] = it.iv + dv[q];
            const bool ok = nb_e[q] >= 0 && nb_e[q] < g.nve && nb_v[q] >= 0 && nb_v[q] < g.nvp;
            if (!ok) nb_e[q] = -1;
            nb_count += ok;
          }
        }
        auto issue_own = [&](int d) {
          const int slot = (int)(og % OWN_SLOTS);
          const unsigned use = og / OWN_SLOTS;
          if (use > 0) alive &= wait_phase(&own_empty[slot], (uint32_t)((use - 1) & 1), timeout);
          if (!alive) return;
          fence_async_shared();
          const int psi = ((it.p0 + d) % g.nh + g.nh) % g.nh;
          mbar_expect_tx(&own_full[slot], own_bytes);
          bulk_load(own + slot * L.own_floats + own_dst,
                    own_src + plane_index(it.iv, it.ie, psi) * PP, own_bytes,
                    &own_full[slot]);
          og++;
        };
        auto issue_nb = [&](int k) {
          const int slot = (int)(ng % NB_SLOTS);
          const unsigned use = ng / NB_SLOTS;
          if (use > 0) alive &= wait_phase(&nb_empty[slot], (uint32_t)((use - 1) & 1), timeout);
          if (!alive) return;
          fence_async_shared();
          mbar_expect_tx(&nb_full[slot], nb_bytes * (nb_count + (BLEND ? 1 : 0)));
          for (int q = 0; q < NEIGHBOURS; q++)
            if (nb_e[q] >= 0)
              bulk_load(nbr + (slot * NB_PLANES + q) * L.nb_floats,
                        a.s.src + plane_index(nb_v[q], nb_e[q], it.p0 + k) * PP +
                            (int64_t)it.y0 * XP,
                        nb_bytes, &nb_full[slot]);
          // the blend partner V of this step's rows: read here before any
          // consumer writes them (they wait for this set first)
          if (BLEND)
            bulk_load(nbr + (slot * NB_PLANES + NEIGHBOURS) * L.nb_floats,
                      a.s.dst + plane_index(it.iv, it.ie, it.p0 + k) * PP +
                          (int64_t)it.y0 * XP,
                      nb_bytes, &nb_full[slot]);
          ng++;
        };
        for (int d = -2; d <= 1 && alive; d++) issue_own(d);
        for (int k = 0; k < it.steps && alive; k++) {
          issue_own(k + 2);
          if (alive) issue_nb(k);
        }
      }
      // Every issued copy is consumed by the consumer warps, which wait for
      // it; after a timeout wait (bounded) for the last one before exiting.
      if (!alive && og > 0)
        wait_phase(&own_full[(og - 1) % OWN_SLOTS], (uint32_t)(((og - 1) / OWN_SLOTS) & 1),
                   timeout);
    }
  } else {
    const int r = tid / a.xc, c = tid % a.xc;
    const int x0 = 4 * c;
    const float ext = (float)g.extent, dxf = (float)g.dx;
    const float ap = (float)g.acc_p, ae = (float)g.acc_e;
    float xs[4];
#pragma unroll
    for (int i = 0; i < 4; i++) xs[i] = fmaf((float)(x0 + i), dxf, -ext);
    const float2 negx_a = make_float2(-xs[0], -xs[1]), negx_b = make_float2(-xs[2], -xs[3]);
    const float2 absx_a = make_float2(fabsf(xs[0]), fabsf(xs[1]));
    const float2 absx_b = make_float2(fabsf(xs[2]), fabsf(xs[3]));
    const float hx = 0.5f * a.ihx, hp = 0.5f * a.ihp, hv = 0.5f * a.ihv, he = 0.5f * a.ihe;
    const float dt = a.dt;
    const bool has_exit = a.s.exit_keep != nullptr;
    const float exit_r = (float)a.s.exit_r;
    const int ctr = (r + 2) * XP + x0;  // this chunk in an own slot
    const int nbo = r * XP + x0;        // this chunk in a neighbour slot
    const bool tail = x0 + 4 > g.nx;                // chunk holds row padding
    float2 finite_acc = f2(0.f);
    unsigned og = 0, ng = 0;

    for (int idx = blockIdx.x; idx < a.items; idx += gridDim.x) {
      const Item it = decode_item(a, idx);
      const bool active = r < it.r_eff;
      const int iy = it.y0 + r;
      const bool y_edge = iy < 2 || iy + 2 >= g.nx;
      const int2 keep = has_exit ? a.s.exit_keep[iy] : make_int2(0, 0);
      const float vp = (float)(g.vp_lo + it.iv * g.dvp);
      const float ve = (float)(g.ve_lo + it.ie * g.dve);
      const float wp = fabsf(vp) * (float)g.curv_p;
      const float we = fabsf(ve) * (float)g.curv_e;
      const float plo = it.iv == 0 ? 0.f : -ap, phi = it.iv == g.nvp - 1 ? 0.f : ap;
      const float elo = it.ie == 0 ? 0.f : -ae, ehi = it.ie == g.nve - 1 ? 0.f : ae;
      const bool p_inner = it.iv > 0 && it.iv < g.nvp - 1;
      const bool e_inner = it.ie > 0 && it.ie < g.nve - 1;
      const bool v_slope_inner = it.iv >= 2 && it.iv + 2 < g.nvp;
      const bool e_slope_inner = it.ie >= 2 && it.ie + 2 < g.nve;
      const float y = fmaf((float)iy, dxf, -ext);
      const float ap_coef = (wp + we) * a.ihp, av_coef = ap * a.ihv, ae_coef = ae * a.ihe;
      const float2 ay_a = __fmul2_rn(__fmul2_rn(f2(wp), absx_a), f2(a.ihx));
      const float2 ay_b = __fmul2_rn(__fmul2_rn(f2(wp), absx_b), f2(a.ihx));
      const float wy = wp * fabsf(y) * a.ihx;
      const int64_t out0 =
          plane_index(it.iv, it.ie, it.p0) * PP + (int64_t)iy * XP + x0;
      float *gdst = a.s.dst + out0;
      float *garr = a.s.arrival + out0;
      const unsigned base = og;  // global index of own plane d = -2

      // Heading window: this chunk at headings k-2 .. k+2.
      float4 win[5];
#pragma unroll
      for (int d = 0; d < 5; d++) {
        const unsigned q = base + d;
        const int slot = (int)(q % OWN_SLOTS);
        if (alive) alive &= wait_phase(&own_full[slot], (uint32_t)((q / OWN_SLOTS) & 1), timeout);
        win[d] = *reinterpret_cast<const float4 *>(own + slot * L.own_floats + ctr);
      }

      // ring positions, advanced by one per step: the refill plane k+2 (slot
      // and phase parity), the centre plane k, the neighbour set
      int rslot = (int)((base + 5) % OWN_SLOTS);  // plane 3, read at k = 1
      uint32_t rpar = (uint32_t)(((base + 5) / OWN_SLOTS) & 1);
      int cslot = (int)((base + 2) % OWN_SLOTS);
      int ns = (int)(ng % NB_SLOTS);
      uint32_t npar = (uint32_t)((ng / NB_SLOTS) & 1);
      for (int k = 0; k < it.steps; k++) {
        if (k > 0) {
          if (alive) alive &= wait_phase(&own_full[rslot], rpar, timeout);
#pragma unroll
          for (int d = 0; d < 4; d++) win[d] = win[d + 1];
          win[4] = *reinterpret_cast<const float4 *>(own + rslot * L.own_floats + ctr);
        }
        if (alive) alive &= wait_phase(&nb_full[ns], npar, timeout);

        if (active && alive) {
          const float *o0 = own + cslot * L.own_floats + ctr;
          const float *nb = nbr + ns * NB_PLANES * L.nb_floats + nbo;
          const float4 C = win[2];
          const float2 v_a = lo2(C), v_b = hi2(C);

          // x: window x0-2 .. x0+5
          const float2 xl = *reinterpret_cast<const float2 *>(o0 - 2);
          const float2 xr = *reinterpret_cast<const float2 *>(o0 + 4);
          const float w[8] = {xl.x, xl.y, C.x, C.y, C.z, C.w, xr.x, xr.y};
          float xlo[4], xhi[4];
          // every warp holds chunks at both x ends: the end rules as selects
          // cost less than running both variants of a divergent branch
          slopes_x<ORDER, true>(w, x0, g.nx, xlo, xhi);
          const float2 lx_a = make_float2(xlo[0], xlo[1]), lx_b = make_float2(xlo[2], xlo[3]);
          const float2 hx_a = make_float2(xhi[0], xhi[1]), hx_b = make_float2(xhi[2], xhi[3]);

          // y: rows iy-2 .. iy+2 of heading k
          float2 ly_a, ly_b, hy_a, hy_b;
          {
            const float4 m2 = *reinterpret_cast<const float4 *>(o0 - 2 * XP);
            const float4 m1 = *reinterpret_cast<const float4 *>(o0 - XP);
            const float4 p1 = *reinterpret_cast<const float4 *>(o0 + XP);
            const float4 p2 = *reinterpret_cast<const float4 *>(o0 + 2 * XP);
            if (y_edge) {
              slope_pair<ORDER, true>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), iy, g.nx, ly_a, hy_a);
              slope_pair<ORDER, true>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), iy, g.nx, ly_b, hy_b);
            } else {
              slope_pair<ORDER, false>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), iy, g.nx, ly_a, hy_a);
              slope_pair<ORDER, false>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), iy, g.nx, ly_b, hy_b);
            }
          }
          // psi: periodic, from the register window
          float2 lp_a, lp_b, hp_a, hp_b;
          slope_pair<ORDER, false>(lo2(win[0]), lo2(win[1]), v_a, lo2(win[3]), lo2(win[4]), 2, 5, lp_a, hp_a);
          slope_pair<ORDER, false>(hi2(win[0]), hi2(win[1]), v_b, hi2(win[3]), hi2(win[4]), 2, 5, lp_b, hp_b);
          // vE and vP: neighbour slots
          float2 le_a, le_b, he_a, he_b, lv_a, lv_b, hv_a, hv_b;
          {
            const float4 m2 = *reinterpret_cast<const float4 *>(nb + 0 * L.nb_floats);
            const float4 m1 = *reinterpret_cast<const float4 *>(nb + 1 * L.nb_floats);
            const float4 p1 = *reinterpret_cast<const float4 *>(nb + 2 * L.nb_floats);
            const float4 p2 = *reinterpret_cast<const float4 *>(nb + 3 * L.nb_floats);
            if (e_slope_inner) {
              slope_pair<ORDER, false>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), it.ie, g.nve, le_a, he_a);
              slope_pair<ORDER, false>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), it.ie, g.nve, le_b, he_b);
            } else {
              slope_pair<ORDER, true>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), it.ie, g.nve, le_a, he_a);
              slope_pair<ORDER, true>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), it.ie, g.nve, le_b, he_b);
            }
          }
          {
            const float4 m2 = *reinterpret_cast<const float4 *>(nb + 4 * L.nb_floats);
            const float4 m1 = *reinterpret_cast<const float4 *>(nb + 5 * L.nb_floats);
            const float4 p1 = *reinterpret_cast<const float4 *>(nb + 6 * L.nb_floats);
            const float4 p2 = *reinterpret_cast<const float4 *>(nb + 7 * L.nb_floats);
            if (v_slope_inner) {
              slope_pair<ORDER, false>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), it.iv, g.nvp, lv_a, hv_a);
              slope_pair<ORDER, false>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), it.iv, g.nvp, lv_b, hv_b);
            } else {
              slope_pair<ORDER, true>(lo2(m2), lo2(m1), v_a, lo2(p1), lo2(p2), it.iv, g.nvp, lv_a, hv_a);
              slope_pair<ORDER, true>(hi2(m2), hi2(m1), v_b, hi2(p1), hi2(p2), it.iv, g.nvp, lv_b, hv_b);
            }
          }

          // Hamiltonian + dissipation (native_relative.cpp:144-157).
          const int ip = it.p0 + k;
          const float bx = fmaf(ve, trig[2 * ip], -vp);
          const float by = ve * trig[2 * ip + 1];
          const float2 bx2 = f2(bx), by2 = f2(by);
          const float ax_coef = fmaf(fabsf(bx), a.ihx, wy);  // alpha_x / h
          const float aby = fabsf(by) * a.ihx;
          const float4 prev4 =
              BLEND ? *reinterpret_cast<const float4 *>(nb + NEIGHBOURS * L.nb_floats) : C;

          float2 out[2];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const float2 lx = h ? lx_b : lx_a, hxv = h ? hx_b : hx_a;
            const float2 ly = h ? ly_b : ly_a, hy = h ? hy_b : hy_a;
            const float2 lp = h ? lp_b : lp_a, hpv = h ? hp_b : hp_a;
            const float2 lv = h ? lv_b : lv_a, hvv = h ? hv_b : hv_a;
            const float2 le = h ? le_b : le_a, hev = h ? he_b : he_a;
            const float2 v = h ? v_b : v_a;
            const float2 negx = h ? negx_b : negx_a;
            const float2 ay = __fadd2_rn(h ? ay_b : ay_a, f2(aby));
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
            }
            if (p_inner) {
#pragma unroll
              for (int l = 0; l < 2; l++) hs[l] = fmaf(-ap, fabsf(gvs[l]), hs[l]);
            } else {
#pragma unroll
              for (int l = 0; l < 2; l++) hs[l] += fminf(plo * gvs[l], phi * gvs[l]);
            }
            if (e_inner) {
#pragma unroll
              for (int l = 0; l < 2; l++) hs[l] = fmaf(ae, fabsf(ges[l]), hs[l]);
            } else {
#pragma unroll
              for (int l = 0; l < 2; l++) hs[l] += fmaxf(elo * ges[l], ehi * ges[l]);
            }
            H = make_float2(hs[0], hs[1]);
            // dissipation: sum alpha_k/h_k * (hi - lo)_k
            float2 diss = __fmul2_rn(f2(ax_coef), sub2(hxv, lx));
            diss = __ffma2_rn(ay, sub2(hy, ly), diss);
            diss = __ffma2_rn(f2(ap_coef), sub2(hpv, lp), diss);
            diss = __ffma2_rn(f2(av_coef), sub2(hvv, lv), diss);
            diss = __ffma2_rn(f2(ae_coef), sub2(hev, le), diss);
            H = __ffma2_rn(f2(0.5f), diss, H);
            float2 value =
                __ffma2_rn(f2(dt), make_float2(fminf(H.x, 0.f), fminf(H.y, 0.f)), v);
            const float2 prev = BLEND ? (h ? hi2(prev4) : lo2(prev4)) : v;
            if (BLEND) value = __fmul2_rn(f2(0.5f), __fadd2_rn(prev, value));
            if (has_exit) {  // cells beyond the local exit hold the exit value
              const int ix = x0 + 2 * h;
              if (ix < keep.x || ix > keep.y) value.x = exit_r;
              if (ix + 1 < keep.x || ix + 1 > keep.y) value.y = exit_r;
            }
            if (tail && x0 + 2 * h + 1 >= g.nx) {  // row padding stays 0
              if (x0 + 2 * h >= g.nx) value.x = 0.f;
              value.y = 0.f;
            }
            finite_acc = __ffma2_rn(value, f2(0.f), finite_acc);
            out[h] = value;
            if (BLEND || ORDER == 1) {
              const float2 change = sub2(value, prev);
              residual = fmaxf(residual, fmaxf(fabsf(change.x), fabsf(change.y)));
              // First crossing of zero (native_relative.cpp:167-168).  The
              // update never increases a cell, so a crossing has
              // prev * value <= 0 with prev > 0.
              const float2 sgn = __fmul2_rn(prev, value);
              if (sgn.x <= 0.f || sgn.y <= 0.f) {
                const float pv[2] = {prev.x, prev.y}, nv[2] = {value.x, value.y};
#pragma unroll
                for (int l = 0; l < 2; l++) {
                  float *slot = garr + 2 * h + l;
                  if (pv[l] > 0.f && nv[l] <= 0.f && x0 + 2 * h + l < g.nx && isnan(*slot))
                    *slot = (float)(a.s.t + a.s.dt * (double)pv[l] /
                                                ((double)pv[l] - (double)nv[l]));
                }
              }
            }
          }
          *reinterpret_cast<float4 *>(gdst) =
              make_float4(out[0].x, out[0].y, out[1].x, out[1].y);
        }
        // Release plane k (and the window-only planes at the item's ends) and
        // this step's neighbour set.
        __syncwarp();
        if (lane == 0) {
          if (k == 0) {
            mbar_arrive(&own_empty[(int)(base % OWN_SLOTS)]);
            mbar_arrive(&own_empty[(int)((base + 1) % OWN_SLOTS)]);
          }
          mbar_arrive(&own_empty[cslot]);
          if (k == it.steps - 1) {
            mbar_arrive(&own_empty[(int)((base + it.steps + 2) % OWN_SLOTS)]);
            mbar_arrive(&own_empty[(int)((base + it.steps + 3) % OWN_SLOTS)]);
          }
          mbar_arrive(&nb_empty[ns]);
        }
        ng++;
        gdst += PP;
        garr += PP;
        if (k > 0 && ++rslot == OWN_SLOTS) {
          rslot = 0;
          rpar ^= 1u;
        }
        if (++cslot == OWN_SLOTS) cslot = 0;
        if (++ns == NB_SLOTS) {
          ns = 0;
          npar ^= 1u;
        }
      }
      og = base + it.steps + 4;
    }
    bad = !(isfinite(finite_acc.x) && isfinite(finite_acc.y));
  }

  // Block reductions: non-finite flag and the largest change.
  if (__syncthreads_or(bad) && tid == 0) atomicOr(&a.s.stats->nonfinite, 1u);
  if (BLEND || ORDER == 1) {
    for (int off = 16; off > 0; off >>= 1)
      residual = fmaxf(residual, __shfl_xor_sync(0xffffffffu, residual, off));
    if (lane == 0) red[warp] = residual;
    __syncthreads();
    if (tid == 0) {
      float m = 0.f;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, red[w]);
      if (m > 0.f)
        atomicMax(&a.s.stats->residual,
                  (unsigned long long)__double_as_longlong((double)m));
    }
  }
}

int g_last_resident = 0;

template <int ORDER, int BLEND>
cudaError_t launch(const FastArgs &args, size_t smem, int threads,
                   cudaStream_t stream) {
  // Resident CTAs per SM for this (shared memory, block size); recomputed
  // when either changes.
  static int configured_smem = 0, configured_threads = 0;
  static int resident = 0;
  if (configured_smem != (int)smem || configured_threads != threads || resident == 0) {
    cudaError_t e = cudaFuncSetAttribute(rel5_stage_kernel<ORDER, BLEND>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &resident, rel5_stage_kernel<ORDER, BLEND>, threads, smem);
    if (e != cudaSuccess) return e;
    if (resident < 1) return cudaErrorInvalidConfiguration;
    configured_smem = (int)smem;
    configured_threads = threads;
  }
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = std::min(args.items, sms * resident);
  g_last_resident = resident;
  rel5_stage_kernel<ORDER, BLEND><<<blocks, threads, smem, stream>>>(args);
  return cudaGetLastError();
}

__global__ void rel5_init_kernel(const float *__restrict__ plane, int64_t plane_size,
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
    // dense index modulo the plane: one (y, x) plane or a (psi, y, x) block
    const int64_t dense = (j / pp) * nx * nx + (int64_t)iy * nx + ix;
    const float v = plane ? plane[dense % plane_size] : field[j];
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

int rel5_last_resident_ctas() { return g_last_resident; }

size_t rel5_fast_smem_bytes(const Rel5Grid &g, const Rel5Tile &t) {
  return (size_t)smem_layout(t.rows, g.xp, g.nh).bytes;
}

Rel5Tile rel5_default_tile(const Rel5Grid &g) {
  const int xc = g.xp / 4;
  Rel5Tile t{1, 8};
  // rows: at most 7 consumer warps, fewest idle rows, then most rows.
  int best_waste = 1 << 30;
  for (int rows = 1; rows * xc <= TARGET_THREADS - 32 && rows <= g.nx; rows++) {
    const int slabs = (g.nx + rows - 1) / rows;
    const int waste = slabs * rows - g.nx;
    if (waste < best_waste || (waste == best_waste && rows > t.rows)) {
      best_waste = waste;
      t.rows = rows;
    }
  }
  // Heading chunks of 24 measured fastest on the 65x48x21x21 grid (B200).
  t.psi_chunk = g.nh < 24 ? g.nh : 24;
  return t;
}

bool rel5_tile_valid(const Rel5Grid &g, const Rel5Tile &t) {
  if (t.rows < 1 || t.rows > g.nx || t.psi_chunk < 1 || t.psi_chunk > g.nh)
    return false;
  const int consumer_warps = (t.rows * (g.xp / 4) + 31) / 32;
  if (32 * (consumer_warps + 1) > TARGET_THREADS) return false;
  return rel5_fast_smem_bytes(g, t) <= 227 * 1024;
}

cudaError_t rel5_stage_f32(const Rel5Grid &g, const Rel5Tile &t,
                           const Rel5Stage &s, int blend, cudaStream_t stream) {
  if (!rel5_tile_valid(g, t)) return cudaErrorInvalidConfiguration;
  FastArgs args;
  args.g = g;
  args.s = s;
  args.rows = t.rows;
  args.psi_chunk = t.psi_chunk;
  args.xc = g.xp / 4;
  args.consumer_warps = (t.rows * args.xc + 31) / 32;
  args.slabs = (g.nx + t.rows - 1) / t.rows;
  args.chunks = (g.nh + t.psi_chunk - 1) / t.psi_chunk;
  args.vp_first = g.own_n > 0 ? g.own_lo : 0;
  args.vp_count = g.own_n > 0 ? g.own_n : g.nvp;
  args.items = args.slabs * g.nve * args.vp_count * args.chunks;
  args.ihx = (float)(1.0 / g.dx);
  args.ihp = (float)(1.0 / g.dphi);
  args.ihv = (float)(1.0 / g.dvp);
  args.ihe = (float)(1.0 / g.dve);
  args.dt = (float)s.dt;
  const int threads = 32 * (args.consumer_warps + 1);
  const size_t smem = rel5_fast_smem_bytes(g, t);
  if (g.order == 1) return launch<1, 0>(args, smem, threads, stream);
  if (blend) return launch<2, 1>(args, smem, threads, stream);
  return launch<2, 0>(args, smem, threads, stream);
}

__global__ void rel5_probe_kernel(const float *__restrict__ field, int nx, int xp,
                                  int64_t n, const int64_t *__restrict__ idx,
                                  const double *__restrict__ w, double *__restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double total = 0;
  for (int k = 0; k < 32; k++) {
    const int64_t d = idx[32 * i + k];  // dense index -> padded row layout
    total += w[32 * i + k] * (double)field[(d / nx) * xp + d % nx];
  }
  out[i] = total;
}

__global__ void rel5_exit_rows_kernel(int nx, float extent, float r2, int2 *keep) {
  const int iy = blockIdx.x * blockDim.x + threadIdx.x;
  if (iy >= nx) return;
  // explicit round-to-nearest operations: nothing is contracted
  const float dx = __fdiv_rn(__fmul_rn(2.f, extent), (float)(nx - 1));
  const float y = __fadd_rn(-extent, __fmul_rn((float)iy, dx));
  const float yy = __fmul_rn(y, y);
  int lo = nx, hi = -1;
  for (int ix = 0; ix < nx; ix++) {
    const float x = __fadd_rn(-extent, __fmul_rn((float)ix, dx));
    if (!(__fadd_rn(__fmul_rn(x, x), yy) > r2)) {
      lo = min(lo, ix);
      hi = ix;
    }
  }
  keep[iy] = make_int2(lo, hi);  // x^2 is unimodal in ix: the kept set is one range
}

cudaError_t rel5_exit_rows(const Rel5Grid &g, float r2, int2 *keep, cudaStream_t stream) {
  rel5_exit_rows_kernel<<<(g.nx + 127) / 128, 128, 0, stream>>>(g.nx, (float)g.extent, r2,
                                                                keep);
  return cudaGetLastError();
}

cudaError_t rel5_probe(const Rel5Grid &g, const float *field, int64_t n, const int64_t *idx,
                       const double *w, double *out, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  rel5_probe_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(field, g.nx, g.xp, n, idx,
                                                                     w, out);
  return cudaGetLastError();
}

cudaError_t rel5_init(const Rel5Grid &g, const float *plane, float *field,
                      float *arrival, float start_time, cudaStream_t stream,
                      int64_t plane_size) {
  const int threads = 256;
  int64_t blocks = (g.n_padded + threads - 1) / threads;
  if (blocks > 148 * 64) blocks = 148 * 64;
  rel5_init_kernel<<<(unsigned)blocks, threads, 0, stream>>>(
      plane, plane_size > 0 ? plane_size : (int64_t)g.nx * g.nx, field, arrival, g.n_padded,
      g.nx, g.xp, start_time);
  return cudaGetLastError();
}

}  // namespace pe
