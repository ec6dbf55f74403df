// Relative 5D ENO/LF stage, fast variant: float32 storage and float32 local
// arithmetic, one launch per RK stage (native_relative.cpp:124-172).
//
// Work decomposition.  A work item is `rows` consecutive y rows of one
// (vP, vE) pair over `psi_chunk` consecutive headings; a persistent CTA walks
// a strided list of items.  A consumer thread owns one 16-byte chunk of 4
// consecutive x cells in one row and walks the item's headings.  For each
// heading step k the CTA needs, in shared memory:
//   * its own (vP, vE) plane at heading k, rows y0-2 .. y0+R+1 (the y halo),
//     for the centre, x and y neighbours, and the plane at heading k+2, from
//     which each thread takes its chunk to extend the heading differences;
//     own planes live in a ring of 8 slots;
//   * the 8 neighbour planes (vE+-1, vE+-2, vP+-1, vP+-2) at heading k, rows
//     y0 .. y0+R-1 (and, on RK2 stage 2, the step's old value V of the same
//     rows), in a ring of 2 neighbour sets.
// All of it arrives by bulk asynchronous copies (the TMA engine,
// cp.async.bulk) issued by a producer warp that runs up to two heading steps
// ahead, across items.  Every copy of step k (the own plane k+2, or planes
// -2..2 on an item's first step, and the neighbour set) completes on that
// step's "full" barrier, and every consumer thread releases the step on its
// "empty" barrier: one wait and one arrival per step.  The ring of 8 own slots makes
// this safe: a plane's slot is refilled two steps after the plane's last use
// (items have at least 4 headings).  Every wait is bounded: a wait that gives
// up sets the handle's timeout flag instead of hanging.
//
// Arithmetic.  The 4 cells of a chunk are processed as two float2 pairs with
// sm_100 packed FP32 instructions (__ffma2_rn / __fadd2_rn / __fmul2_rn).
// Second differences are kept unscaled (h^2 * D2) and the ENO2 slopes are
// (first difference +- 0.5 * selected second difference) / h -- the
// reference's dm + 0.5*h*D2 rewritten.  Along the heading axis the first
// and second differences and the ENO selection of an edge are computed once
// and carried to the next heading (the low-side slope of heading k+1 is
// formed with the high-side selection of heading k).  Along x the
// differences and selections are shared between the cells of a chunk, and
// the end rules sit at compile-time positions (nx mod 4).  Each axis'
// slopes enter the update only as their sum (the centred gradient times 2h)
// and their jump (hi - lo, the Lax-Friedrichs term), so the 1/(2h) scalings
// are folded into per-item and per-heading coefficients.  Results agree with
// the double-local reference to float rounding except where an ENO selection
// is tied to rounding; relative5d_exact.cu is the bit-exact path.
#include <algorithm>
#include <cstdio>

#include "bulk_copy.cuh"
#include "relative5d.cuh"
#include "relative5d_eno_f32.cuh"

namespace pe {
namespace {

using namespace eno32;
using namespace bulk;

constexpr int OWN_SLOTS = 8;   // own-plane ring (power of two)
constexpr int STEP_SLOTS = 2;  // neighbour sets and step barriers
constexpr int NEIGHBOURS = 8;  // vE-2, vE-1, vE+1, vE+2, vP-2, vP-1, vP+1, vP+2
// a neighbour set also holds, on RK2 stage 2, the item's rows of the
// stage's old value V (the blend partner), prefetched with the neighbours
constexpr int NB_PLANES = NEIGHBOURS + 1;
constexpr int MAX_THREADS = 512;
constexpr int TARGET_THREADS = 256;  // launch bound: two CTAs of 256 per SM
constexpr int MIN_ITEM_STEPS = 4;    // own-ring reuse needs items of >= 4 headings
// A try waits for up to the hardware's own time limit before it returns
// false; a wait gives up after WAIT_LIMIT tries.  (On the 89M-cell grid a
// suspend-time hint of 1 us per try measured 0.8 % slower, and a
// %globaltimer bound in the loop 1.3 % slower.)
constexpr unsigned WAIT_LIMIT = 1u << 21;

// Bounded wait for one mbarrier phase.  Returns false (and flags the handle)
// when the limit is reached.
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t parity,
                                           unsigned int *timeout_flag) {
  return bulk::wait_phase(bar, parity, timeout_flag, WAIT_LIMIT);
}

struct FastArgs {
  Rel5Grid g;
  Rel5Stage s;
  int rows, psi_chunk, slabs, chunks, xc, consumer_warps, items;
  int vp_first, vp_count;  // the vP slabs this launch updates (a shard's own)
  float ihx, ihp, ihv, ihe;
  float dt;
};

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
  L.bar_off = 4 * (L.nb_off + STEP_SLOTS * NB_PLANES * L.nb_floats);
  L.red_off = L.bar_off + 8 * 2 * STEP_SLOTS;
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

__device__ __forceinline__ float2 ld2(const float *p) {
  return *reinterpret_cast<const float2 *>(p);
}
__device__ __forceinline__ float4 ld4(const float *p) {
  return *reinterpret_cast<const float4 *>(p);
}

// Sum and jump (hi + lo, hi - lo) of the ENO slopes of two cells along a
// non-walked axis from their five values.
template <int ORDER, bool GENERAL>
__device__ __forceinline__ void sum_jump(float2 m2, float2 m1, float2 v, float2 p1, float2 p2,
                                         int pos, int n, float2 &S, float2 &J) {
  float2 lo, hi;
  slope_pair<ORDER, GENERAL>(m2, m1, v, p1, p2, pos, n, lo, hi);
  S = add2(lo, hi);
  J = sub2(hi, lo);
}

// The same for the 4 cells of a chunk (two pairs) along a vertical or speed
// axis, from the chunks of the four neighbouring nodes.
template <int ORDER, bool GENERAL>
__device__ __forceinline__ void sum_jump4(float4 m2, float4 m1, float4 v, float4 p1, float4 p2,
                                          int pos, int n, float2 S[2], float2 J[2]) {
  sum_jump<ORDER, GENERAL>(lo2(m2), lo2(m1), lo2(v), lo2(p1), lo2(p2), pos, n, S[0], J[0]);
  sum_jump<ORDER, GENERAL>(hi2(m2), hi2(m1), hi2(v), hi2(p1), hi2(p2), pos, n, S[1], J[1]);
}


// Persistent, warp-specialised stage kernel.  Each CTA walks the items
// blockIdx.x, blockIdx.x + gridDim.x, ...  Warps 0..consumer_warps-1 compute
// 4-cell chunks; the last warp is the producer: its lane 0 issues every bulk
// copy in the order the consumers need them, across item boundaries.  Own
// planes of an item are numbered d = -2 .. steps+1 and take ring slots in
// issue order: plane d of an item whose first plane was the og-th issued
// sits in slot (og + d + 2) mod 8.  Plane d is read at step d (centre, x and
// y neighbours) and at step d-2 (heading differences); planes -2..1 only
// start the item's heading differences at step 0.
//
// XR = nx mod 4 places the x end rules (see slopes_x_fixed).
template <int ORDER, int BLEND, int XR, int XPC, int RC>
__global__ void __launch_bounds__(TARGET_THREADS, 2)
    rel5_stage_kernel(const FastArgs a) {
  extern __shared__ __align__(128) float smem[];
  const Rel5Grid &g = a.g;
  // XPC / RC: the row pitch and tile rows at compile time (0: from the
  // arguments), so that every shared-memory offset is an immediate
  const int R = RC ? RC : a.rows, XP = XPC ? XPC : g.xp;
  const int XC = XPC ? XPC / 4 : a.xc;
  const SmemLayout L = smem_layout(R, XP, g.nh);
  float *own = smem + L.own_off;  // [8][R+4][XP]
  float *nbr = smem + L.nb_off;   // [2][9][R][XP]
  char *raw = reinterpret_cast<char *>(smem);
  uint64_t *full = reinterpret_cast<uint64_t *>(raw + L.bar_off);
  uint64_t *empty = full + STEP_SLOTS;
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
    for (int i = 0; i < STEP_SLOTS; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 32 * a.consumer_warps);
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
      unsigned og = 0, gs = 0;  // own planes / steps issued so far
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
        for (int k = 0; k < it.steps; k++) {
          const int slot = (int)(gs & 1u);
          // the slot's previous step (gs - 2) must be released first
          if (gs >= STEP_SLOTS)
            alive = wait_phase(&empty[slot], ((gs >> 1) - 1) & 1u, timeout);
          if (!alive) break;
          fence_async_shared();
          const int d_first = k == 0 ? -2 : k + 2;
          const int n_own = k + 3 - d_first;
          mbar_expect_tx(&full[slot], (uint32_t)n_own * own_bytes +
                                          nb_bytes * (nb_count + (BLEND ? 1 : 0)));
          for (int d = d_first; d <= k + 2; d++) {
            const int psi = ((it.p0 + d) % g.nh + g.nh) % g.nh;
            bulk_load(own + (og & (OWN_SLOTS - 1)) * L.own_floats + own_dst,
                      own_src + plane_index(it.iv, it.ie, psi) * PP, own_bytes, &full[slot]);
            og++;
          }
          float *set = nbr + slot * NB_PLANES * L.nb_floats;
          for (int q = 0; q < NEIGHBOURS; q++)
            if (nb_e[q] >= 0)
              bulk_load(set + q * L.nb_floats,
                        a.s.src + plane_index(nb_v[q], nb_e[q], it.p0 + k) * PP +
                            (int64_t)it.y0 * XP,
                        nb_bytes, &full[slot]);
          // the blend partner V of this step's rows: read here before any
          // consumer writes them (they wait for this set first)
          if (BLEND)
            bulk_load(set + NEIGHBOURS * L.nb_floats,
                      a.s.dst + plane_index(it.iv, it.ie, it.p0 + k) * PP +
                          (int64_t)it.y0 * XP,
                      nb_bytes, &full[slot]);
          gs++;
        }
      }
      // After a timeout, let the copies already issued (the last two steps'
      // sets at most) land before the CTA exits.
      if (!alive)
        for (unsigned q = gs > STEP_SLOTS ? gs - STEP_SLOTS : 0; q < gs; q++)
          wait_phase(&full[q & 1u], (q >> 1) & 1u, timeout);
    }
  } else {
    const int r = tid / XC, c = tid % XC;
    const int x0 = 4 * c;
    const float ext = (float)g.extent, dxf = (float)g.dx;
    const float ap = (float)g.acc_p, ae = (float)g.acc_e;
    // half reciprocal spacings: a centred gradient is (lo + hi) * h?s
    const float hxs = 0.5f * a.ihx, hps = 0.5f * a.ihp, hvs = 0.5f * a.ihv, hes = 0.5f * a.ihe;
    float xs[4];
#pragma unroll
    for (int i = 0; i < 4; i++) xs[i] = fmaf((float)(x0 + i), dxf, -ext);
    // -x * hxs per cell (the -x*gy term of y*gx - x*gy - gp), |x| per cell
    const float2 nxs[2] = {make_float2(-xs[0] * hxs, -xs[1] * hxs),
                           make_float2(-xs[2] * hxs, -xs[3] * hxs)};
    const float2 absx[2] = {make_float2(fabsf(xs[0]), fabsf(xs[1])),
                            make_float2(fabsf(xs[2]), fabsf(xs[3]))};
    constexpr int IEND = (XR + 3) & 3;
    constexpr int KEND = XR >= 2 ? XR : XR + 4;
    const bool first = x0 == 0;
    const bool kend_chunk = x0 == g.nx - KEND;
    const bool iend_chunk = x0 == g.nx - 1 - IEND;
    const float dt = a.dt;
    const bool has_exit = a.s.exit_keep != nullptr;
    const float exit_r = (float)a.s.exit_r;
    const int ctr = (r + 2) * XP + x0;  // this chunk in an own slot
    const int nbo = r * XP + x0;        // this chunk in a neighbour slot
    float2 finite_acc = f2(0.f);
    unsigned og = 0, gs = 0;

    for (int idx = blockIdx.x; idx < a.items && alive; idx += gridDim.x) {
      const Item it = decode_item(a, idx);
      const bool active = r < it.r_eff;
      const int iy = it.y0 + r;
      // warps holding a row within two of a y end take the general y rules
      // (warp-uniform: the warp's first and last active rows)
      const int rw0 = (32 * warp) / XC;
      const int rw1 = min((32 * warp + 31) / XC, it.r_eff - 1);
      const bool y_general = it.y0 + rw0 < 2 || it.y0 + rw1 + 2 >= g.nx;
      const int2 keep = has_exit && active ? a.s.exit_keep[iy] : make_int2(0, 0);
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
      const float ys = y * hxs;
      // Coefficients of the update, per item.  The Hamiltonian is
      //   bx*gx + by*gy - wp*|y*gx - x*gy - gp| + we*|gp| + speed terms
      // with g = (lo + hi) * h?s, and the Lax-Friedrichs term
      //   sum_axis alpha_axis * h?s * (hi - lo)
      // with alpha = |bx| + wp|y|, |by| + wp|x|, wp + we, ap, ae.
      const float wes = we * hps;                       // * |S_psi|
      const float kv_in = -ap * hvs, ke_in = ae * hes;  // * |S_v|, |S_e| (inner)
      const float dap = (wp + we) * hps, dav = ap * hvs, dae = ae * hes;
      const float dax0 = wp * fabsf(y) * hxs;  // + |bx| * hxs per heading
      const float2 day0[2] = {__fmul2_rn(f2(wp * hxs), absx[0]),
                              __fmul2_rn(f2(wp * hxs), absx[1])};  // + |by| * hxs
      const unsigned base = og;  // issue index of own plane d = -2
      og += it.steps + 4;
      const int64_t out0 = plane_index(it.iv, it.ie, it.p0) * PP + (int64_t)iy * XP + x0;
      float *gdst = a.s.dst + out0;
      float *garr = a.s.arrival + out0;
      auto own_at = [&](unsigned q) -> const float * {
        return own + (q & (OWN_SLOTS - 1)) * L.own_floats + ctr;
      };

      // Step 0's set holds planes -2..2: start the heading differences.
      if (alive) alive = wait_phase(&full[gs & 1u], (gs >> 1) & 1u, timeout);
      // carried along the headings, per pair of cells: VN = V(k+1),
      // ER = V(k+1) - V(k), D2 = second difference at k (ORDER 2), LO = low
      // slope of heading k
      float2 VN[2], ER[2], D2[2], LO[2];
      if (active) {  // lanes past the item's rows read nothing
        const float4 vm2 = ld4(own_at(base)), vm1 = ld4(own_at(base + 1));
        const float4 v0 = ld4(own_at(base + 2)), vp1 = ld4(own_at(base + 3));
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const float2 a_m2 = h ? hi2(vm2) : lo2(vm2), a_m1 = h ? hi2(vm1) : lo2(vm1);
          const float2 a_0 = h ? hi2(v0) : lo2(v0), a_p1 = h ? hi2(vp1) : lo2(vp1);
          const float2 el = sub2(a_0, a_m1);
          ER[h] = sub2(a_p1, a_0);
          VN[h] = a_p1;
          if (ORDER == 1) {
            LO[h] = el;
            D2[h] = f2(0.f);
          } else {
            const float2 dm = sub2(el, sub2(a_m1, a_m2));
            D2[h] = sub2(ER[h], el);
            LO[h] = __ffma2_rn(f2(0.5f), pick2(dm, D2[h]), el);
          }
        }
      }

      // one step per iteration: unrolling by two spills on stage 1 and the
      // local-memory traffic costs more than the saved register moves
#pragma unroll 1
      for (int k = 0; k < it.steps; k++) {
        const unsigned slot = gs & 1u;
        if (k > 0 && alive) alive = wait_phase(&full[slot], (gs >> 1) & 1u, timeout);
        if (active && alive) {
          const float *o0 = own_at(base + k + 2);  // centre plane k
          const float *nb = nbr + slot * NB_PLANES * L.nb_floats + nbo;
          const float4 C = ld4(o0);
          const float4 VNEW = ld4(own_at(base + k + 4));  // plane k+2

          // heading k: cos, sin
          const float cs_k = trig[2 * (it.p0 + k)], sn_k = trig[2 * (it.p0 + k) + 1];
          const float bx = fmaf(ve, cs_k, -vp), by = ve * sn_k;
          const float cx = bx * hxs, cy = by * hxs;
          const float dax = fmaf(fabsf(bx), hxs, dax0);
          const float aby = fabsf(by) * hxs;

          // Accumulators per pair: A and D = linear terms and dissipation
          // (x and y; heading and speeds: two shorter dependency chains),
          // T = y*gx - x*gy - gp, Hs = the absolute-value and speed terms
          // (scalar FMAs take |S| as an operand).
          float2 A[2], D[2], T[2];
          float Hs[2][2];

          // x: window x0-2 .. x0+5 (end rules at compile-time positions)
          {
            const float2 xl = ld2(o0 - 2), xr = ld2(o0 + 4);
            const float w[8] = {xl.x, xl.y, C.x, C.y, C.z, C.w, xr.x, xr.y};
            float xlo[4], xhi[4];
            slopes_x_fixed<ORDER, XR>(w, first, kend_chunk, iend_chunk, xlo, xhi);
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const float2 lo = make_float2(xlo[2 * h], xlo[2 * h + 1]);
              const float2 hi = make_float2(xhi[2 * h], xhi[2 * h + 1]);
              const float2 S = add2(lo, hi), J = sub2(hi, lo);
              A[h] = __ffma2_rn(f2(dax), J, __fmul2_rn(f2(cx), S));
              T[h] = __fmul2_rn(f2(ys), S);
            }
          }
          // y: rows iy-2 .. iy+2 of heading k
          {
            const float4 m2 = ld4(o0 - 2 * XP), m1 = ld4(o0 - XP);
            const float4 p1 = ld4(o0 + XP), p2 = ld4(o0 + 2 * XP);
            float2 S[2], J[2];
            if (y_general)
              sum_jump4<ORDER, true>(m2, m1, C, p1, p2, iy, g.nx, S, J);
            else
              sum_jump4<ORDER, false>(m2, m1, C, p1, p2, iy, g.nx, S, J);
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const float2 day = __fadd2_rn(day0[h], f2(aby));
              A[h] = __ffma2_rn(f2(cy), S[h], A[h]);
              A[h] = __ffma2_rn(day, J[h], A[h]);
              T[h] = __ffma2_rn(nxs[h], S[h], T[h]);
            }
          }
          // psi: extend the carried differences with heading k+2
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const float2 vnew = h ? hi2(VNEW) : lo2(VNEW);
            const float2 en = sub2(vnew, VN[h]);  // V(k+2) - V(k+1)
            float2 hi, lo_next;
            if (ORDER == 1) {
              hi = ER[h];
              lo_next = ER[h];
            } else {
              const float2 d2n = sub2(en, ER[h]);
              const float2 pr = pick2(D2[h], d2n);
              hi = __ffma2_rn(f2(-0.5f), pr, ER[h]);
              lo_next = __ffma2_rn(f2(0.5f), pr, ER[h]);
              D2[h] = d2n;
            }
            const float2 S = add2(LO[h], hi), J = sub2(hi, LO[h]);
            LO[h] = lo_next;
            ER[h] = en;
            VN[h] = vnew;
            T[h] = __ffma2_rn(f2(-hps), S, T[h]);
            D[h] = __fmul2_rn(f2(dap), J);
            Hs[h][0] = wes * fabsf(S.x);
            Hs[h][1] = wes * fabsf(S.y);
          }
          // vE and vP: neighbour planes
          {
            const float4 m2 = ld4(nb + 0 * L.nb_floats), m1 = ld4(nb + 1 * L.nb_floats);
            const float4 p1 = ld4(nb + 2 * L.nb_floats), p2 = ld4(nb + 3 * L.nb_floats);
            float2 S[2], J[2];
            if (e_slope_inner)
              sum_jump4<ORDER, false>(m2, m1, C, p1, p2, it.ie, g.nve, S, J);
            else
              sum_jump4<ORDER, true>(m2, m1, C, p1, p2, it.ie, g.nve, S, J);
#pragma unroll
            for (int h = 0; h < 2; h++) {
              D[h] = __ffma2_rn(f2(dae), J[h], D[h]);
              if (e_inner) {
                Hs[h][0] = fmaf(ke_in, fabsf(S[h].x), Hs[h][0]);
                Hs[h][1] = fmaf(ke_in, fabsf(S[h].y), Hs[h][1]);
              } else {  // max(elo*ge, ehi*ge), ge = S * hes
                const float2 ge = __fmul2_rn(f2(hes), S[h]);
                Hs[h][0] += fmaxf(elo * ge.x, ehi * ge.x);
                Hs[h][1] += fmaxf(elo * ge.y, ehi * ge.y);
              }
            }
          }
          {
            const float4 m2 = ld4(nb + 4 * L.nb_floats), m1 = ld4(nb + 5 * L.nb_floats);
            const float4 p1 = ld4(nb + 6 * L.nb_floats), p2 = ld4(nb + 7 * L.nb_floats);
            float2 S[2], J[2];
            if (v_slope_inner)
              sum_jump4<ORDER, false>(m2, m1, C, p1, p2, it.iv, g.nvp, S, J);
            else
              sum_jump4<ORDER, true>(m2, m1, C, p1, p2, it.iv, g.nvp, S, J);
#pragma unroll
            for (int h = 0; h < 2; h++) {
              D[h] = __ffma2_rn(f2(dav), J[h], D[h]);
              if (p_inner) {
                Hs[h][0] = fmaf(kv_in, fabsf(S[h].x), Hs[h][0]);
                Hs[h][1] = fmaf(kv_in, fabsf(S[h].y), Hs[h][1]);
              } else {  // min(plo*gv, phi*gv), gv = S * hvs
                const float2 gv = __fmul2_rn(f2(hvs), S[h]);
                Hs[h][0] += fminf(plo * gv.x, phi * gv.x);
                Hs[h][1] += fminf(plo * gv.y, phi * gv.y);
              }
            }
          }

          const float4 prev4 = BLEND ? ld4(nb + NEIGHBOURS * L.nb_floats) : C;
          float2 out[2];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const float2 v = h ? hi2(C) : lo2(C);
            // H = A + D + Hs - wp * |T|
            const float2 Hs2 = make_float2(fmaf(-wp, fabsf(T[h].x), Hs[h][0]),
                                           fmaf(-wp, fabsf(T[h].y), Hs[h][1]));
            const float2 Hsum = __fadd2_rn(__fadd2_rn(A[h], D[h]), Hs2);
            float2 value =
                __ffma2_rn(f2(dt), make_float2(fminf(Hsum.x, 0.f), fminf(Hsum.y, 0.f)), v);
            const float2 prev = BLEND ? (h ? hi2(prev4) : lo2(prev4)) : v;
            if (BLEND) value = __fmul2_rn(f2(0.5f), __fadd2_rn(prev, value));
            if (has_exit) {  // cells beyond the local exit hold the exit value
              const int ix = x0 + 2 * h;
              if (ix < keep.x || ix > keep.y) value.x = exit_r;
              if (ix + 1 < keep.x || ix + 1 > keep.y) value.y = exit_r;
            }
            out[h] = value;
          }
          if (iend_chunk) {  // row padding past x = nx-1 stays 0
            if (IEND < 1) out[0].y = 0.f;
            if (IEND < 2) out[1].x = 0.f;
            if (IEND < 3) out[1].y = 0.f;
          }
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const float2 value = out[h];
            finite_acc = __ffma2_rn(value, f2(0.f), finite_acc);
            if (BLEND || ORDER == 1) {
              const float2 prev = BLEND ? (h ? hi2(prev4) : lo2(prev4)) : (h ? hi2(C) : lo2(C));
              const float2 change = sub2(value, prev);
              residual = fmaxf(residual, fmaxf(fabsf(change.x), fabsf(change.y)));
              // First crossing of zero (native_relative.cpp:167-168).  The
              // update never increases a cell, so a crossing has
              // prev * value <= 0 with prev > 0; padding holds 0 and never
              // crosses.
              const float2 sgn = __fmul2_rn(prev, value);
              if (sgn.x <= 0.f || sgn.y <= 0.f) {
                const float pv[2] = {prev.x, prev.y}, nv[2] = {value.x, value.y};
#pragma unroll
                for (int l = 0; l < 2; l++) {
                  float *slot_p = garr + 2 * h + l;
                  if (pv[l] > 0.f && nv[l] <= 0.f && isnan(*slot_p))
                    *slot_p = (float)(a.s.t + a.s.dt * (double)pv[l] /
                                                  ((double)pv[l] - (double)nv[l]));
                }
              }
            }
          }
          *reinterpret_cast<float4 *>(gdst) =
              make_float4(out[0].x, out[0].y, out[1].x, out[1].y);
        }
        // Release this step's set (and the own planes it finished): each
        // thread after its own reads, so no lane waits on another.
        mbar_arrive(&empty[slot]);
        gs++;
        gdst += PP;
        garr += PP;
      }
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

template <int ORDER, int BLEND, int XR, int XPC = 0, int RC = 0>
cudaError_t launch_xr(const FastArgs &args, size_t smem, int threads, cudaStream_t stream) {
  // Resident CTAs per SM for this (shared memory, block size); recomputed
  // when either changes.
  static int configured_smem = 0, configured_threads = 0;
  static int resident = 0;
  if (configured_smem != (int)smem || configured_threads != threads || resident == 0) {
    cudaError_t e = cudaFuncSetAttribute(rel5_stage_kernel<ORDER, BLEND, XR, XPC, RC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &resident, rel5_stage_kernel<ORDER, BLEND, XR, XPC, RC>, threads, smem);
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
  rel5_stage_kernel<ORDER, BLEND, XR, XPC, RC><<<blocks, threads, smem, stream>>>(args);
  return cudaGetLastError();
}

template <int ORDER, int BLEND>
cudaError_t launch(const FastArgs &args, size_t smem, int threads, cudaStream_t stream) {
  // the 65-position grids (68-float rows) at the default 13-row tile, with
  // compile-time offsets (5 % faster on the 89M-cell grid, B200)
  if (args.g.xp == 68 && args.g.nx == 65 && args.rows == 13)
    return launch_xr<ORDER, BLEND, 1, 68, 13>(args, smem, threads, stream);
  switch (args.g.nx & 3) {
    case 0: return launch_xr<ORDER, BLEND, 0>(args, smem, threads, stream);
    case 1: return launch_xr<ORDER, BLEND, 1>(args, smem, threads, stream);
    case 2: return launch_xr<ORDER, BLEND, 2>(args, smem, threads, stream);
    default: return launch_xr<ORDER, BLEND, 3>(args, smem, threads, stream);
  }
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
  // Heading chunks of about 24 (fastest on the 65x48x21x21 grid, B200),
  // balanced so that the last chunk is not short.
  const int chunks = (g.nh + 23) / 24;
  t.psi_chunk = (g.nh + chunks - 1) / chunks;
  return t;
}

bool rel5_tile_valid(const Rel5Grid &g, const Rel5Tile &t) {
  if (t.rows < 1 || t.rows > g.nx || t.psi_chunk < 1 || t.psi_chunk > g.nh)
    return false;
  // every item (the last heading chunk too) needs MIN_ITEM_STEPS headings
  const int tail = g.nh % t.psi_chunk;
  if (t.psi_chunk < MIN_ITEM_STEPS || (tail != 0 && tail < MIN_ITEM_STEPS)) return false;
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
