// Batched relative 5D solves with the float32 cell update, tiled: the
// formulas of the exact update (native_relative.cpp:38-67 slopes, :124-172
// stage) in float32 with reciprocal spacings and multiply-add contraction,
// the arithmetic of the single-grid float32 kernel (relative5d_fast.cu).
//
// A work item is `rows` y rows of one (vP, vE) plane stack of one solve, all
// headings.  A thread owns a 4-cell x chunk of one row and walks the
// headings, carrying the heading differences and ENO selections from one
// heading to the next (the psi stencil).  For each heading the CTA stages,
// double-buffered against the previous heading's arithmetic, the item's own
// plane rows with a 2-row y halo and the rows of the 8 speed-neighbour
// planes (vE +-1, +-2, vP +-1, +-2): lanes 0-8 of warp 0 issue one bulk
// copy (cp.async.bulk, the TMA engine) each, one per contiguous row range,
// all completing on the buffer's mbarrier, on which every thread waits
// (bounded); the x, y and speed stencils then read shared
// memory.  The persistent loop over steps, the active-item prefix and the
// bounded grid barrier are those of relative5d_batch_impl.cuh.
#include "bulk_copy.cuh"
#include "relative5d_batch_impl.cuh"
#include "relative5d_eno_f32.cuh"

namespace pe {
namespace {

using namespace eno32;

constexpr int kThreads = kRel5BatchThreads;
constexpr int kNb = 8;  // vE-2, vE-1, vE+1, vE+2, vP-2, vP-1, vP+1, vP+2
// tries of a bounded wait for a staged heading
constexpr unsigned kStageWaitLimit = 1u << 22;

// The two heading buffers' mbarriers, and the flag a wait that gives up
// raises (set once per launch).
__shared__ uint64_t stage_bar[2];
__shared__ unsigned *stage_timeout;

// Fill state of the two heading buffers, the same in every thread of the
// CTA: bit b = number of fills of buffer b mod 2, bit 2 + b = buffer b was
// filled at least once.
struct StageRing {
  unsigned bits = 0;
  // parity of the mbarrier phase of buffer b's latest fill
  __device__ __forceinline__ unsigned parity(int b) const { return ((bits >> b) & 1u) ^ 1u; }
  __device__ __forceinline__ void filled(int b) { bits = (bits ^ (1u << b)) | (4u << b); }
  __device__ __forceinline__ bool used(int b) const { return (bits >> (2 + b)) & 1u; }
};

__device__ __forceinline__ void wait_staged(const StageRing &ring, int b) {
  for (unsigned i = 0; i < kStageWaitLimit; i++)
    if (bulk::mbar_try_wait(&stage_bar[b], ring.parity(b))) return;
  atomicOr(stage_timeout, 1u);
}

// Shared memory of one heading: own rows [R + 4][xp] then [kNb][R][xp].
__host__ __device__ inline int buffer_floats(int rows, int xp) {
  return (rows + 4) * xp + kNb * rows * xp;
}

struct ItemGeom {
  int iv, ie, y0, r_eff, R, xc;
};

// Stage heading `psi` of an item into buffer `buf` (called by warp 0): the
// own plane rows y0-2 .. y0+r_eff+1 inside the box (lane 8) and rows
// y0 .. y0+r_eff-1 of each speed-neighbour plane inside the grid (lane q for
// neighbour q), each a contiguous range (rows are xp floats, xp a multiple
// of 4, so every range starts and ends on 16 bytes), completing on `bar`.
// Lane 0 first posts the byte count of all of them.
__device__ __forceinline__ void stage_heading(const Rel5Grid &g, const float *__restrict__ src,
                                              const ItemGeom &it, int psi, float *buf,
                                              uint64_t *bar) {
  const int lane = threadIdx.x & 31;
  const int xp = g.xp;
  const int64_t PP = (int64_t)g.nx * xp;
  const uint32_t nb_bytes = (uint32_t)(it.r_eff * xp * 4);
  const int lo = max(0, it.y0 - 2), hi = min(g.nx, it.y0 + it.r_eff + 2);
  const uint32_t own_bytes = (uint32_t)((hi - lo) * xp * 4);
  if (lane == 0) {
    // speed neighbours inside the grid: vE-2..vE+2 and vP-2..vP+2 minus the
    // centre, cut at the ends
    const int count = min(it.ie + 2, g.nve - 1) - max(it.ie - 2, 0) +
                      min(it.iv + 2, g.nvp - 1) - max(it.iv - 2, 0);
    bulk::mbar_expect_tx(bar, own_bytes + (uint32_t)count * nb_bytes);
  }
  __syncwarp();
  if (lane < kNb) {
    const int d = (lane & 3) < 2 ? (lane & 3) - 2 : (lane & 3) - 1;  // -2, -1, +1, +2
    const int nv = it.iv + (lane < 4 ? 0 : d), ne = it.ie + (lane < 4 ? d : 0);
    if (nv >= 0 && nv < g.nvp && ne >= 0 && ne < g.nve) {
      bulk::fence_async_shared();
      bulk::bulk_load(buf + (it.R + 4 + lane * it.R) * xp,
                      src + (((int64_t)nv * g.nve + ne) * g.nh + psi) * PP + (int64_t)it.y0 * xp,
                      nb_bytes, bar);
    }
  } else if (lane == kNb) {
    bulk::fence_async_shared();
    bulk::bulk_load(buf + (lo - it.y0 + 2) * xp,
                    src + (((int64_t)it.iv * g.nve + it.ie) * g.nh + psi) * PP + (int64_t)lo * xp,
                    own_bytes, bar);
  }
}

// One stage of one item (all headings).  Returns the largest |change| of
// this thread's cells (stage 2) and flags non-finite values.
template <int ORDER, int BLEND>
__device__ __forceinline__ void item_stage(const Rel5Grid &g, const Rel5Stage &s,
                                           const ItemGeom &it, float *smem, StageRing &ring,
                                           float &change_max, float &change_up,
                                           float2 &finite_acc) {
  const int xp = g.xp, xc = it.xc;
  const int64_t PP = (int64_t)g.nx * xp;
  const int tid = threadIdx.x;
  const int r = tid / xc, c = tid - (tid / xc) * xc;
  const bool active = tid < it.R * xc && r < it.r_eff;
  const int x0 = 4 * c, iy = it.y0 + r;
  const int bufsz = buffer_floats(it.R, xp);

  const float ext = (float)g.extent, dxf = (float)g.dx;
  const float ihx = (float)(1.0 / g.dx), ihp = (float)(1.0 / g.dphi);
  const float ihv = (float)(1.0 / g.dvp), ihe = (float)(1.0 / g.dve);
  const float ap = (float)g.acc_p, ae = (float)g.acc_e;
  const float vp = (float)(g.vp_lo + it.iv * g.dvp), ve = (float)(g.ve_lo + it.ie * g.dve);
  const float wp = fabsf(vp) * (float)g.curv_p, we = fabsf(ve) * (float)g.curv_e;
  const float plo = it.iv == 0 ? 0.f : -ap, phi = it.iv == g.nvp - 1 ? 0.f : ap;
  const float elo = it.ie == 0 ? 0.f : -ae, ehi = it.ie == g.nve - 1 ? 0.f : ae;
  const bool p_inner = it.iv > 0 && it.iv < g.nvp - 1;
  const bool e_inner = it.ie > 0 && it.ie < g.nve - 1;
  const bool v_slope_inner = it.iv >= 2 && it.iv + 2 < g.nvp;
  const bool e_slope_inner = it.ie >= 2 && it.ie + 2 < g.nve;
  const bool y_edge = iy < 2 || iy + 2 >= g.nx;
  const bool tail = x0 + 4 > g.nx;
  float xs[4];
#pragma unroll
  for (int i = 0; i < 4; i++) xs[i] = fmaf((float)(x0 + i), dxf, -ext);
  // half reciprocal spacings: a centred gradient is (lo + hi) * h?s, so each
  // axis enters the update through the sum S = lo + hi and the jump
  // J = hi - lo of its slopes (the single-grid float32 kernel's arithmetic)
  const float hxs = 0.5f * ihx, hps = 0.5f * ihp, hvs = 0.5f * ihv, hes = 0.5f * ihe;
  const float2 nxs[2] = {make_float2(-xs[0] * hxs, -xs[1] * hxs),
                         make_float2(-xs[2] * hxs, -xs[3] * hxs)};
  const float2 day0[2] = {make_float2(wp * hxs * fabsf(xs[0]), wp * hxs * fabsf(xs[1])),
                          make_float2(wp * hxs * fabsf(xs[2]), wp * hxs * fabsf(xs[3]))};
  const float dt = (float)s.dt;
  const float y = fmaf((float)iy, dxf, -ext);
  const float ys = y * hxs;
  const float wes = we * hps;                       // * |S_psi|
  const float kv_in = -ap * hvs, ke_in = ae * hes;  // * |S_v|, |S_e| (inner)
  const float dap = (wp + we) * hps, dav = ap * hvs, dae = ae * hes;
  const float dax0 = wp * fabsf(y) * hxs;  // + |bx| * hxs per heading
  const int64_t stack = ((int64_t)it.iv * g.nve + it.ie) * g.nh * PP;
  const int64_t cell0 = stack + (int64_t)iy * xp + x0;  // heading 0
  const int nh = g.nh;
  auto wrap = [nh](int q) { return q < 0 ? q + nh : (q >= nh ? q - nh : q); };
  auto load_plane = [&](int q) {
    return active ? *reinterpret_cast<const float4 *>(s.src + cell0 + (int64_t)wrap(q) * PP)
                  : make_float4(0.f, 0.f, 0.f, 0.f);
  };

  // The heading axis is walked: its differences and ENO selection are
  // carried from one heading to the next, per pair of cells.  VN = V(k+1),
  // ER = V(k+1) - V(k), D2 = second difference at k, LO = low slope at k;
  // C = V(k), VNEW = V(k+2), `next` = V(k+3) (one heading ahead, from L2).
  float2 VN[2], ER[2], D2[2], LO[2];
  float4 C, VNEW;
  {
    const float4 vm2 = load_plane(-2), vm1 = load_plane(-1), v0 = load_plane(0);
    const float4 vp1 = load_plane(1);
    VNEW = load_plane(2);
    C = v0;
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

  if (tid < 32) stage_heading(g, s.src, it, 0, smem, &stage_bar[0]);
  ring.filled(0);
  for (int k = 0; k < nh; k++) {
    const int b = k & 1;
    wait_staged(ring, b);
    __syncthreads();  // heading k staged; heading k-1's buffer no longer read
    if (k + 1 < nh) {
      if (tid < 32)
        stage_heading(g, s.src, it, k + 1, smem + (b ^ 1) * bufsz, &stage_bar[b ^ 1]);
      ring.filled(b ^ 1);
    }
    const float4 next = k + 1 < nh ? load_plane(k + 3) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float *own = smem + b * bufsz;
    if (active) {
      const float *o0 = own + (r + 2) * xp + x0;
      const float *nb = own + (it.R + 4) * xp + r * xp + x0;
      const float bx = fmaf(ve, (float)s.cs[k], -vp), by = ve * (float)s.sn[k];
      const float cx = bx * hxs, cy = by * hxs;
      const float dax = fmaf(fabsf(bx), hxs, dax0);
      const float aby = fabsf(by) * hxs;
      // A: linear terms and x/y dissipation, D: heading and speed
      // dissipation, T = y gx - x gy - gp, Hs: absolute-value and speed terms
      float2 A[2], D[2], T[2];
      float Hs[2][2];
      {  // x: window x0-2 .. x0+5 of the padded row
        const float2 xl = *reinterpret_cast<const float2 *>(o0 - 2);
        const float2 xr = *reinterpret_cast<const float2 *>(o0 + 4);
        // rows are padded: x0 - 2 < 0 and x0 + 5 >= xp only read the row's
        // neighbours in the buffer, which the end rules of slopes_x ignore
        const float w[8] = {xl.x, xl.y, C.x, C.y, C.z, C.w, xr.x, xr.y};
        float xlo[4], xhi[4];
        slopes_x<ORDER, true>(w, x0, g.nx, xlo, xhi);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const float2 lo = make_float2(xlo[2 * h], xlo[2 * h + 1]);
          const float2 hi = make_float2(xhi[2 * h], xhi[2 * h + 1]);
          const float2 S = add2(lo, hi), J = sub2(hi, lo);
          A[h] = __ffma2_rn(f2(dax), J, __fmul2_rn(f2(cx), S));
          T[h] = __fmul2_rn(f2(ys), S);
        }
      }
      {  // y: rows iy-2 .. iy+2 of heading k
        const float4 m2 = *reinterpret_cast<const float4 *>(o0 - 2 * xp);
        const float4 m1 = *reinterpret_cast<const float4 *>(o0 - xp);
        const float4 p1 = *reinterpret_cast<const float4 *>(o0 + xp);
        const float4 p2 = *reinterpret_cast<const float4 *>(o0 + 2 * xp);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          float2 lo, hi;
          const float2 c2 = h ? hi2(C) : lo2(C);
          if (y_edge)
            slope_pair<ORDER, true>(h ? hi2(m2) : lo2(m2), h ? hi2(m1) : lo2(m1), c2,
                                    h ? hi2(p1) : lo2(p1), h ? hi2(p2) : lo2(p2), iy, g.nx,
                                    lo, hi);
          else
            slope_pair<ORDER, false>(h ? hi2(m2) : lo2(m2), h ? hi2(m1) : lo2(m1), c2,
                                     h ? hi2(p1) : lo2(p1), h ? hi2(p2) : lo2(p2), iy, g.nx,
                                     lo, hi);
          const float2 S = add2(lo, hi), J = sub2(hi, lo);
          const float2 day = __fadd2_rn(day0[h], f2(aby));
          A[h] = __ffma2_rn(f2(cy), S, A[h]);
          A[h] = __ffma2_rn(day, J, A[h]);
          T[h] = __ffma2_rn(nxs[h], S, T[h]);
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
        T[h] = __ffma2_rn(f2(-hps), S, T[h]);
        D[h] = __fmul2_rn(f2(dap), J);
        Hs[h][0] = wes * fabsf(S.x);
        Hs[h][1] = wes * fabsf(S.y);
      }
      const int nbf = it.R * xp;
      {  // vE: neighbour planes 0-3
        const float4 m2 = *reinterpret_cast<const float4 *>(nb + 0 * nbf);
        const float4 m1 = *reinterpret_cast<const float4 *>(nb + 1 * nbf);
        const float4 p1 = *reinterpret_cast<const float4 *>(nb + 2 * nbf);
        const float4 p2 = *reinterpret_cast<const float4 *>(nb + 3 * nbf);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          float2 lo, hi;
          const float2 c2 = h ? hi2(C) : lo2(C);
          if (e_slope_inner)
            slope_pair<ORDER, false>(h ? hi2(m2) : lo2(m2), h ? hi2(m1) : lo2(m1), c2,
                                     h ? hi2(p1) : lo2(p1), h ? hi2(p2) : lo2(p2), it.ie,
                                     g.nve, lo, hi);
          else
            slope_pair<ORDER, true>(h ? hi2(m2) : lo2(m2), h ? hi2(m1) : lo2(m1), c2,
                                    h ? hi2(p1) : lo2(p1), h ? hi2(p2) : lo2(p2), it.ie,
                                    g.nve, lo, hi);
          const float2 S = add2(lo, hi), J = sub2(hi, lo);
          D[h] = __ffma2_rn(f2(dae), J, D[h]);
          if (e_inner) {
            Hs[h][0] = fmaf(ke_in, fabsf(S.x), Hs[h][0]);
            Hs[h][1] = fmaf(ke_in, fabsf(S.y), Hs[h][1]);
          } else {  // max(elo*ge, ehi*ge), ge = S * hes
            const float2 ge = __fmul2_rn(f2(hes), S);
            Hs[h][0] += fmaxf(elo * ge.x, ehi * ge.x);
            Hs[h][1] += fmaxf(elo * ge.y, ehi * ge.y);
          }
        }
      }
      {  // vP: neighbour planes 4-7
        const float4 m2 = *reinterpret_cast<const float4 *>(nb + 4 * nbf);
        const float4 m1 = *reinterpret_cast<const float4 *>(nb + 5 * nbf);
        const float4 p1 = *reinterpret_cast<const float4 *>(nb + 6 * nbf);
        const float4 p2 = *reinterpret_cast<const float4 *>(nb + 7 * nbf);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          float2 lo, hi;
          const float2 c2 = h ? hi2(C) : lo2(C);
          if (v_slope_inner)
            slope_pair<ORDER, false>(h ? hi2(m2) : lo2(m2), h ? hi2(m1) : lo2(m1), c2,
                                     h ? hi2(p1) : lo2(p1), h ? hi2(p2) : lo2(p2), it.iv,
                                     g.nvp, lo, hi);
          else
            slope_pair<ORDER, true>(h ? hi2(m2) : lo2(m2), h ? hi2(m1) : lo2(m1), c2,
                                    h ? hi2(p1) : lo2(p1), h ? hi2(p2) : lo2(p2), it.iv,
                                    g.nvp, lo, hi);
          const float2 S = add2(lo, hi), J = sub2(hi, lo);
          D[h] = __ffma2_rn(f2(dav), J, D[h]);
          if (p_inner) {
            Hs[h][0] = fmaf(kv_in, fabsf(S.x), Hs[h][0]);
            Hs[h][1] = fmaf(kv_in, fabsf(S.y), Hs[h][1]);
          } else {  // min(plo*gv, phi*gv), gv = S * hvs
            const float2 gv = __fmul2_rn(f2(hvs), S);
            Hs[h][0] += fminf(plo * gv.x, phi * gv.x);
            Hs[h][1] += fminf(plo * gv.y, phi * gv.y);
          }
        }
      }
      const int64_t cell = cell0 + (int64_t)k * PP;
      const float4 prev4 = BLEND ? *reinterpret_cast<const float4 *>(s.dst + cell) : C;
      float2 out[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const float2 v = h ? hi2(C) : lo2(C);
        // H = A + D + Hs - wp * |T|
        const float2 Hs2 = make_float2(fmaf(-wp, fabsf(T[h].x), Hs[h][0]),
                                       fmaf(-wp, fabsf(T[h].y), Hs[h][1]));
        const float2 H = __fadd2_rn(__fadd2_rn(A[h], D[h]), Hs2);
        float2 value = __ffma2_rn(f2(dt), make_float2(fminf(H.x, 0.f), fminf(H.y, 0.f)), v);
        const float2 prev = BLEND ? (h ? hi2(prev4) : lo2(prev4)) : v;
        if (BLEND) value = __fmul2_rn(f2(0.5f), __fadd2_rn(prev, value));
        if (tail && x0 + 2 * h + 1 >= g.nx) {  // row padding stays 0
          if (x0 + 2 * h >= g.nx) value.x = 0.f;
          value.y = 0.f;
        }
        finite_acc = __ffma2_rn(value, f2(0.f), finite_acc);
        out[h] = value;
        if (BLEND) {
          const float2 change = sub2(value, prev);
          change_max = fmaxf(change_max, fmaxf(fabsf(change.x), fabsf(change.y)));
          change_up = fmaxf(change_up, fmaxf(change.x, change.y));
          const float2 sgn = __fmul2_rn(prev, value);
          if (sgn.x <= 0.f || sgn.y <= 0.f) {
            const float pv[2] = {prev.x, prev.y}, nv[2] = {value.x, value.y};
#pragma unroll
            for (int l = 0; l < 2; l++) {
              float *slot = s.arrival + cell + 2 * h + l;
              if (pv[l] > 0.f && nv[l] <= 0.f && x0 + 2 * h + l < g.nx && isnan(*slot))
                *slot = (float)(s.t + s.dt * (double)pv[l] /
                                            ((double)pv[l] - (double)nv[l]));
            }
          }
        }
      }
      *reinterpret_cast<float4 *>(s.dst + cell) =
          make_float4(out[0].x, out[0].y, out[1].x, out[1].y);
    }
    // advance the heading window: the next centre is V(k+1), carried in VN
    C = make_float4(VN[0].x, VN[0].y, VN[1].x, VN[1].y);
#pragma unroll
    for (int h = 0; h < 2; h++) VN[h] = h ? hi2(VNEW) : lo2(VNEW);
    VNEW = next;
  }
  __syncthreads();  // the buffers are restaged by the next item
}

template <int BLEND>
__device__ __forceinline__ void tiled_stage(const Rel5BatchArgs &A, int step, int64_t n_items, double *scratch,
                            Rel5Grid *sg, float *smem, StageRing &ring) {
  int64_t lo = 0, hi = 0;
  const Rel5BatchSolve *S = nullptr;
  Rel5Stage s{};
  int rows = 1, slabs = 1, xc = 1;
  float change_max = 0.f, change_up = 0.f;
  float2 finite_acc = make_float2(0.f, 0.f);
  auto flush = [&]() {
    if (!S) return;
    const bool bad = !(isfinite(finite_acc.x) && isfinite(finite_acc.y));
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&S->stats->nonfinite, 1u);
    if (BLEND) {
      const double m_abs = batch_impl::block_max((double)change_max, scratch);
      const double m_up = batch_impl::block_max((double)change_up, scratch);
      if (threadIdx.x == 0) {
        batch_impl::atomic_max_nonneg(&S->stats->residual, m_abs);
        batch_impl::atomic_max_nonneg(&S->stats->increase, m_up);
      }
    }
    change_max = change_up = 0.f;
    finite_acc = make_float2(0.f, 0.f);
  };
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (item < lo || item >= hi) {  // the same for every thread of the CTA
      flush();
      S = &A.solves[batch_impl::find_solve(A, item)];
      lo = S->item_base;
      hi = lo + S->items;
      __syncthreads();  // the previous solve's grid copy is no longer read
      if (threadIdx.x == 0) *sg = S->g;
      const double2 td = S->steps[step];
      s.src = BLEND ? S->b : S->a;
      s.dst = BLEND ? S->a : S->b;
      s.arrival = S->arrival;
      s.sn = S->sn;
      s.cs = S->cs;
      s.t = td.x;
      s.dt = td.y;
      s.stats = S->stats;
      rows = S->rows;
      __syncthreads();
      slabs = (sg->nx + rows - 1) / rows;
      xc = sg->xp / 4;
    }
    const Rel5Grid &g = *sg;
    int64_t local = item - lo;
    ItemGeom it;
    const int slab = (int)(local % slabs);
    local /= slabs;
    it.ie = (int)(local % g.nve);
    it.iv = (int)(local / g.nve);
    it.R = rows;
    it.xc = xc;
    it.y0 = slab * rows;
    it.r_eff = min(rows, g.nx - it.y0);
    item_stage<2, BLEND>(g, s, it, smem, ring, change_max, change_up, finite_acc);
  }
  flush();
}

__global__ void __launch_bounds__(kThreads, 2)
    rel5_batch_tiled_kernel(const Rel5BatchArgs A) {
  extern __shared__ __align__(16) float smem[];
  __shared__ double scratch[kThreads / 32];
  __shared__ Rel5Grid sg;
  if (threadIdx.x == 0) {
    bulk::mbar_init(&stage_bar[0], 1);
    bulk::mbar_init(&stage_bar[1], 1);
    bulk::fence_barrier_init();
    // a stage wait that gives up raises the grid barrier's flag: every CTA
    // leaves at its next barrier and the host reports the timeout
    stage_timeout = &A.sync[2];
  }
  __syncthreads();
  StageRing ring;
  unsigned round = 0;
  for (int step = 0; step < A.max_steps; step++) {
    const int64_t n_items = A.active_items[step];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < A.count;
         k += gridDim.x * blockDim.x)
      if (step < A.solves[k].nsteps) A.solves[k].stats->residual = 0ull;
    tiled_stage<0>(A, step, n_items, scratch, &sg, smem, ring);
    if (!batch_impl::grid_barrier(A.sync, ++round)) break;
    // the next stage's bulk copies read what other CTAs stored before the
    // barrier: order it for the async proxy (warp 0 issues the copies)
    if (threadIdx.x < 32) bulk::fence_async_global();
    tiled_stage<1>(A, step, n_items, scratch, &sg, smem, ring);
    if (!batch_impl::grid_barrier(A.sync, ++round)) break;
    if (threadIdx.x < 32) bulk::fence_async_global();
  }
  // no bulk copy may still be landing when the CTA exits (complete already
  // unless a wait gave up)
  if (threadIdx.x == 0) {
    if (ring.used(0)) wait_staged(ring, 0);
    if (ring.used(1)) wait_staged(ring, 1);
  }
}

}  // namespace

int rel5_batch_tiled_rows(int nx, int xp, int want) {
  const int cap = kThreads / (xp / 4);
  int rows = want < 1 ? cap : want;
  rows = rows > cap ? cap : rows;
  rows = rows > nx ? nx : rows;
  return rows < 1 ? 1 : rows;
}

size_t rel5_batch_tiled_smem(int rows, int xp) {
  return 2 * sizeof(float) * (size_t)buffer_floats(rows, xp);
}

int rel5_batch_grid_tiled(size_t smem) {
  int device = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return 0;
  if (cudaFuncSetAttribute(rel5_batch_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rel5_batch_tiled_kernel, kThreads,
                                                    smem) != cudaSuccess)
    return 0;
  return sms * per_sm;
}

cudaError_t rel5_batch_run_tiled(const Rel5BatchArgs &args, int grid, size_t smem,
                                 cudaStream_t stream) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, rel5_batch_tiled_kernel, args);
}

}  // namespace pe
