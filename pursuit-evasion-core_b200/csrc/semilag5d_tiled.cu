// Relative 5D semi-Lagrangian min-max backup, shared-memory tiled form.
//
// Same semantics as sl_backup_kernel (semilag5d.cu), restructured for
// throughput.  A persistent CTA owns a work item: one (vP, vE) speed pair,
// `rows` y rows at full x width, and a run of headings psi.  The speed
// interpolation of every successor only mixes the three vP and three vE
// slabs around the item, with weights that depend on the acceleration
// alone, so the item stages, for each of the 9 (pursuer accel, evader
// accel) combinations, the speed-blended (y, x) planes of three consecutive
// headings in shared memory (rows + 4 by 72 positions, with two halo cells
// on every side holding the linear extension of the field beyond the
// position box).  They are kept as two "heading-pair" planes of float2:
// (psi-1, psi) and (psi, psi+1), the lower and upper heading of a successor
// side by side.  Every (pursuer, evader) action pair is then a bilinear
// gather of 4 float2 corners (both heading planes at once) plus a heading
// lerp: 4 shared-memory loads instead of 32 global ones, with the position
// lerps in packed FP32.
//
// The ring advances one heading per psi step: the raw slab rows of the
// plane after next are fetched with cp.async while the current heading is
// computed, extended into the halo, blended, and written with the plane
// before it as the new heading pair over the pair that is no longer needed.
//
// Value-only backups prune with the optimal (pursuer, evader) pair of the
// previous backup at each cell (a hint byte) as the guide: a pursuer action
// is abandoned as soon as one evader reply is at least as bad as the best
// value so far -- it can no longer lower the minimum (the reference's
// pruning rule, local_game/grid_game.py:226).  The three evaluation phases
// are described at minmax_cell; min and max are exact, so the value does
// not depend on the visiting order.
//
// The grid holds as many CTAs as fit on the SMs at once (one for the
// default tile, two for tiles of about 6 rows).
//
// Preconditions (checked on the host): nx + 4 <= 72, every successor within
// 1.99 cells of its cell in x and y, heading shifts below one plane, and
// speed successors inside the three staged slabs.
#include "semilag5d.cuh"

namespace pe {
namespace {

constexpr int kPitch = 72;  // ring / raw row pitch in floats
constexpr int kHalo = 2;
constexpr int kCombos = 9;
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: x + kMagic rounds x to an integer
constexpr unsigned kMagicBits = 0x4B400000u;
constexpr int kCPT = 2;  // cells per thread
// Tiles have at most kRowsMax rows, so every staged plane has the fixed
// stride kPlane and all ring and raw offsets are compile-time multiples.
constexpr int kRowsMax = 13;
constexpr int kRR = kRowsMax + 2 * kHalo;  // staged rows of a plane
constexpr int kPlane = kRR * kPitch;       // positions per staged plane

struct __align__(16) SLPair {  // one (pursuer, evader) action pair at the current heading
  float2 o;        // successor offset in local ring coordinates
  float2 cc;       // (c, c), (s, s): the pursuer's turn, successor =
  float2 ss;       //   c (X, Y) + s (Y, -X) + o
  float wp;        // heading weight of the upper plane
  unsigned base;   // float2 offset of its heading-pair plane, minus the
                   // magic bits of the packed (row, col) index
};
static_assert(sizeof(SLPair) == 32, "pair table entry is 32 bytes");

__device__ __forceinline__ int wrap_psi(int q, int nh) {
  const int r = q % nh;
  return r < 0 ? r + nh : r;
}

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)),
               "l"(src)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ float2 sub2(float2 a, float2 b) {  // a - b
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}

// Interpolated value of one action pair at a cell with centred index
// coordinates P = (X, Y) and Q = (Y, -X).  Both position axes, and the two
// heading planes (the .x and .y of every ring element), are carried side by
// side in packed FP32 pairs.
__device__ __forceinline__ float pair_value(const float2 *ring, const SLPair &p, float2 P,
                                            float2 Q) {
  const float2 F = __ffma2_rn(p.cc, P, __ffma2_rn(p.ss, Q, p.o));
  // round(F - 0.5) + magic: the floor of F in the low mantissa bits
  const float2 T = __fadd2_rn(__fadd2_rn(F, make_float2(-0.5f, -0.5f)),
                              make_float2(kMagic, kMagic));
  const float2 W = sub2(F, __fadd2_rn(T, make_float2(-kMagic, -kMagic)));
  const unsigned idx = __float_as_uint(T.y) * (unsigned)kPitch + __float_as_uint(T.x) + p.base;
  const float2 *a = ring + idx;
  const float2 v00 = a[0], v01 = a[1], v10 = a[kPitch], v11 = a[kPitch + 1];
  const float2 wx = make_float2(W.x, W.x), wy = make_float2(W.y, W.y);
  const float2 r0 = __ffma2_rn(wx, sub2(v01, v00), v00);
  const float2 r1 = __ffma2_rn(wx, sub2(v11, v10), v10);
  const float2 r = __ffma2_rn(wy, sub2(r1, r0), r0);
  return fmaf(p.wp, r.y - r.x, r.x);
}

// Value of the raw slab plane at global (gx, gy), extended linearly from the
// edge cell beyond the position box (the reference's clamped-node,
// extrapolated-weight interpolation, reversible/relative_table.py:76-102).
__device__ __forceinline__ float extended(const float *raw_plane, int gx, int gy, int n,
                                          int ty0) {
  // raw_plane rows are local (gy - ty0 + kHalo), columns local (gx + kHalo)
  auto at = [&](int x, int y) {
    return raw_plane[(y - ty0 + kHalo) * kPitch + x + kHalo];
  };
  auto row = [&](int y) {
    if (gx >= 0 && gx < n) return at(gx, y);
    const int cx = gx < 0 ? 0 : n - 2;
    const float v0 = at(cx, y), v1 = at(cx + 1, y);
    return fmaf((float)(gx - cx), v1 - v0, v0);
  };
  if (gy >= 0 && gy < n) return row(gy);
  const int cy = gy < 0 ? 0 : n - 2;
  const float r0 = row(cy), r1 = row(cy + 1);
  return fmaf((float)(gy - cy), r1 - r0, r0);
}

// Pruned min over pursuer actions of the max over evader replies at one
// cell (centred index coordinates P = (X, Y), Q = (Y, -X)), guided by the
// previous backup's optimal pair (hu, he).  `best` enters as the value to
// beat (the current value for the tube, +inf otherwise) and leaves as the
// min-max if that is lower; (bu, be) is then its pair, else (hu, he).
// `live` false skips the work (the warp-wide loops still take part).
//  P.  probe every pursuer action against reply he (9 independent
//      evaluations); an action whose probe already reaches `best` cannot
//      lower the minimum and is dropped;
//  C1. evaluate the other 8 replies of the most promising remaining action
//      (hu if it remains, else the lowest probe) in full;
//  C2. the remaining actions one reply at a time (he first), each abandoned
//      once its reply maximum reaches `best`.
__device__ __forceinline__ void minmax_cell(const float2 *ring, const SLPair *pairs, float2 P,
                                            float2 Q, int hu, int he, bool live, float &best,
                                            int &bu, int &be, unsigned &evals) {
  bu = hu;
  be = he;
  evals += live ? 9u : 0u;
  float probe[9];
#pragma unroll
  for (int u = 0; u < 9; u++) probe[u] = pair_value(ring, pairs[u * 9 + he], P, Q);
  unsigned cand = 0;
  float lo = INFINITY;
  int arg = hu;
#pragma unroll
  for (int u = 0; u < 9; u++) {
    const bool keep = probe[u] < best;
    cand |= keep ? 1u << u : 0u;
    if (keep && probe[u] < lo) {
      lo = probe[u];
      arg = u;
    }
  }
  if (!live) cand = 0;
  const int first = (cand >> hu) & 1u ? hu : arg;
  // C1
  if (__any_sync(0xffffffffu, cand != 0)) {
    evals += cand ? 8u : 0u;
    float w = probe[0];
#pragma unroll
    for (int u = 1; u < 9; u++) w = first == u ? probe[u] : w;
    int wa = he;
#pragma unroll
    for (int j = 0; j < 9; j++) {
      if (j == he) continue;
      const float v = pair_value(ring, pairs[first * 9 + j], P, Q);
      if (v > w) {
        w = v;
        wa = j;
      }
    }
    if (cand && w < best) {
      best = w;
      bu = first;
      be = wa;
    }
    cand &= ~(1u << first);
    unsigned keep = 0;
#pragma unroll
    for (int u = 0; u < 9; u++) keep |= probe[u] < best ? 1u << u : 0u;
    cand &= keep;
  }
  // C2
  int up = cand ? __ffs(cand) - 1 : 0, uj = 0, wue = he;
  float worst = -INFINITY;
  while (__any_sync(0xffffffffu, cand != 0)) {
    if (!cand) continue;
    const int ue = uj == 0 ? he : uj - (uj <= he);
    const float v = pair_value(ring, pairs[up * 9 + ue], P, Q);
    evals++;
    if (v > worst) {
      worst = v;
      wue = ue;
    }
    if (worst >= best || ++uj == 9) {
      if (worst < best) {
        best = worst;
        bu = up;
        be = wue;
      }
      cand &= ~(1u << up);
      up = cand ? __ffs(cand) - 1 : 0;
      uj = 0;
      worst = -INFINITY;
    }
  }
}

template <int MODE, int CPT>
__global__ void __launch_bounds__(SL_TILED_MAX_THREADS, 1)
    sl_tiled_kernel(const SLGrid g, const SLBackup b, const SLTiled t,
                    const SLTiledPlan plan) {
  extern __shared__ __align__(16) float smem[];
  constexpr int pl = kPlane;
  // heading-pair planes [combo][q & 1][rr][kPitch] of float2: the pair
  // (q, q+1) (plane q in .x, q+1 in .y) lives in slot q & 1
  float2 *ring = reinterpret_cast<float2 *>(smem);
  float *raw = smem + 2 * 2 * kCombos * pl;  // [slab][rr][kPitch]
  SLPair *pairs = reinterpret_cast<SLPair *>(raw + kCombos * pl);
  __shared__ int64_t slab_off[kCombos];

  const int nx = g.nx, nh = g.nh;
  const int tid = threadIdx.x, nthreads = blockDim.x;
  const float center = 0.5f * (float)(nx - 1);
  const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;
  float change = 0.f;
  bool bad = false;
  unsigned long long evals_total = 0;

  for (int64_t item = blockIdx.x; item < plan.items; item += gridDim.x) {
    int64_t rest = item;
    const int tile = (int)(rest % plan.tiles_y);
    rest /= plan.tiles_y;
    const int ie = (int)(rest % g.nve);
    rest /= g.nve;
    const int iv = (int)(rest % g.nvp);
    const int chunk = (int)(rest / g.nvp);
    const int ty0 = tile * plan.rows;
    const int trows = min(plan.rows, nx - ty0);
    const int p0 = chunk * plan.psi_chunk, p1 = min(nh, p0 + plan.psi_chunk);
    const SLSpeedStep ps = t.pstep[iv], es = t.estep[ie];
    const int gy_lo = max(0, ty0 - kHalo), gy_hi = min(nx, ty0 + trows + kHalo);
    // this thread's cells of every heading plane of the item: row << 16 |
    // column, or -1 past the tile
    int cpos[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) {
      const int c = tid + k * nthreads;
      const int row = c / nx;
      cpos[k] = c < trows * nx ? (row << 16) | (c - row * nx) : -1;
    }
    const int64_t item_base = (((int64_t)iv * g.nve + ie) * nh) * nx * nx + (int64_t)ty0 * nx;
    if (t.changed_in) {
      // the neighbourhood's flags (the same for every thread: uniform)
      unsigned dirty = 0;
      for (int dv = -1; dv <= 1; dv++)
        for (int de = -1; de <= 1; de++)
          for (int dtile = -1; dtile <= 1; dtile++) {
            const int v = iv + dv, e = ie + de, q = tile + dtile;
            if (v < 0 || v >= g.nvp || e < 0 || e >= g.nve || q < 0 || q >= plan.tiles_y)
              continue;
            dirty |= t.changed_in[((int64_t)chunk * g.nvp + v) * g.nve * plan.tiles_y +
                                  (int64_t)e * plan.tiles_y + q];
          }
      if (!dirty) {  // same inputs as the previous backup: same outputs
        const int span = trows * nx;
        for (int ip = p0; ip < p1; ip++) {
          const int64_t base = item_base + (int64_t)ip * nx * nx;
          for (int c = tid; c < span; c += nthreads) b.dst[base + c] = b.src[base + c];
        }
        if (t.changed_out && tid == 0) t.changed_out[item] = 0;
        continue;
      }
    }
    bool item_changed = false;
    // offsets of the 9 staged (vP, vE) slabs at heading 0
    if (tid < kCombos) {
      const int va = ps.base + tid / 3, vb = es.base + tid % 3;
      slab_off[tid] = ((int64_t)va * g.nve + vb) * nh * nx * nx;
    }
    __syncthreads();

    // raw slab rows of heading plane q (unwrapped) -> raw, asynchronously;
    // one warp per (slab, row), lanes along x
    auto load_raw = [&](int q) {
      const float *plane_src = b.src + (int64_t)wrap_psi(q, nh) * nx * nx;
      for (int rw = warp; rw < kCombos * kRR; rw += nwarps) {
        const int s = rw / kRR, gy = ty0 - kHalo + (rw - s * kRR);
        if (gy < gy_lo || gy >= gy_hi) continue;
        const float *src = plane_src + slab_off[s] + gy * nx + lane;
        float *dst = raw + s * pl + (gy - ty0 + kHalo) * kPitch + kHalo + lane;
#pragma unroll
        for (int i = 0; i < (kPitch - 2 * kHalo + 31) / 32; i++)  // nx <= kPitch - 4
          if (lane + 32 * i < nx) cp_async4(dst + 32 * i, src + 32 * i);
      }
    };
    // halo of the raw plane (needs the in-box rows in place): the two
    // columns on each side of an in-box row (one thread per slab, row and
    // column), whole rows beyond the box (lanes along x)
    auto fill_halo = [&]() {
      const int srows = trows + 2 * kHalo;
      constexpr int side = kCombos * kRR * 2 * kHalo;
      for (int k = tid; k < side; k += nthreads) {
        const int s = k / (kRR * 2 * kHalo), r = k - s * (kRR * 2 * kHalo);
        const int gy = ty0 - kHalo + r / (2 * kHalo), q = r % (2 * kHalo);
        if (gy < gy_lo || gy >= gy_hi) continue;
        const int gx = q < kHalo ? q - kHalo : nx + q - kHalo;
        float *plane = raw + s * pl;
        plane[(gy - ty0 + kHalo) * kPitch + gx + kHalo] = extended(plane, gx, gy, nx, ty0);
      }
      if (ty0 >= kHalo && ty0 + trows + kHalo <= nx) return;  // no row beyond the box
      for (int rw = warp; rw < kCombos * kRR; rw += nwarps) {
        const int s = rw / kRR, lr = rw - s * kRR;
        const int gy = ty0 - kHalo + lr;
        if (lr >= srows || (gy >= 0 && gy < nx)) continue;
        float *plane = raw + s * pl;
        for (int lc = lane; lc < nx + 2 * kHalo; lc += 32)
          plane[lr * kPitch + lc] = extended(plane, lc - kHalo, gy, nx, ty0);
      }
    };
    // speed blends of the raw plane of heading q (whole rows of the pitch:
    // the pad columns past nx + 4 hold unused values, never read).  MODE
    // 0 (warm-up): write the plane as .x of pair (q, q+1) if `as_lower` and
    // as .y of pair (q-1, q) if `as_upper`; MODE 1 (advance): write pair
    // (q-1, q) whole, its .x copied from the .y of pair (q-2, q-1).
    auto blend = [&](int q, bool as_lower, bool as_upper, bool advance) {
      const int count = (trows + 2 * kHalo) * kPitch;
      float2 *lower = ring + (q & 1) * pl;        // pair (q, q+1), combo 0
      float2 *upper = ring + ((q - 1) & 1) * pl;  // pair (q-1, q), combo 0
      const float2 *prev = ring + ((q - 2) & 1) * pl;  // pair (q-2, q-1)
      for (int off = tid; off < count; off += nthreads) {
        float v[9];
#pragma unroll
        for (int s = 0; s < 9; s++) v[s] = raw[s * pl + off];
        float pv[3][3];  // [pursuer accel][evader slab]
#pragma unroll
        for (int a = 0; a < 3; a++) {
          const int lo = ps.slot[a];
          const float w = ps.w[a];
#pragma unroll
          for (int e = 0; e < 3; e++) {
            const float x0 = lo == 0 ? v[e] : v[3 + e];
            const float x1 = lo == 0 ? v[3 + e] : v[6 + e];
            // x0 + w (x1 - x0): equal speeds blend to the value itself, bit
            // for bit, so an unchanged neighbourhood backs up unchanged
            pv[a][e] = fmaf(w, x1 - x0, x0);
          }
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int e = 0; e < 3; e++) {
            const int lo = es.slot[e];
            const float w = es.w[e];
            const float x0 = lo == 0 ? pv[a][0] : pv[a][1];
            const float x1 = lo == 0 ? pv[a][1] : pv[a][2];
            const float nv = fmaf(w, x1 - x0, x0);
            const int c = (a * 3 + e) * 2 * pl + off;
            if (advance) {
              upper[c] = make_float2(prev[c].y, nv);
            } else {
              if (as_lower) reinterpret_cast<float *>(lower + c)[0] = nv;
              if (as_upper) reinterpret_cast<float *>(upper + c)[1] = nv;
            }
          }
      }
    };
    // pair table of heading ip
    auto pair_table = [&](int ip) {
      for (int k = tid; k < 81; k += nthreads) {  // small tiles have < 81 threads
        const int up = k / 9, ue = k % 9;
        const SLPursuerArc pa = b.parc[iv * 9 + up];
        const SLEvaderArc ea = b.earc[ie * 9 + ue];
        const SLEvaderMove em = b.emove[((int64_t)wrap_psi(ip, nh) * g.nve + ie) * 9 + ue];
        const float dxp = em.ex - pa.px, dyp = em.ey - pa.py;
        SLPair p;
        p.o = make_float2(fmaf(pa.c, dxp, pa.s * dyp) * g.ihx + center + (float)kHalo,
                          fmaf(pa.c, dyp, -pa.s * dxp) * g.ihx + center + (float)(kHalo - ty0));
        p.cc = make_float2(pa.c, pa.c);
        p.ss = make_float2(pa.s, pa.s);
        const float delta = ea.turn_idx - pa.turn_idx;
        const float fl = floorf(delta);
        p.wp = delta - fl;
        const int combo = (up / 3) * 3 + ue / 3;
        const int q = ip + (int)fl;  // lower heading of the successor
        const unsigned bias = kMagicBits * (unsigned)(kPitch + 1);
        p.base = (unsigned)((combo * 2 + (q & 1)) * pl) - bias;
        pairs[k] = p;
      }
    };

    // warm-up: planes p0-1, p0, p0+1 into the pairs (p0-1, p0), (p0, p0+1)
    for (int q = p0 - 1; q <= p0 + 1; q++) {
      load_raw(q);
      cp_async_commit_wait();
      __syncthreads();
      fill_halo();
      if (q == p0 + 1) pair_table(p0);
      __syncthreads();
      blend(q, q <= p0, q >= p0, false);
      __syncthreads();
    }
    if (p0 + 2 <= p1) load_raw(p0 + 2);
    cp_async_commit();

    for (int ip = p0; ip < p1; ip++) {
      // ---- compute the cells of heading ip (one cell of each thread at a time)
      const int64_t plane_base = item_base + (int64_t)ip * nx * nx;
#pragma unroll 1
      for (int k = 0; k < CPT; k++) {
        const bool valid = cpos[k] >= 0;
        const int row = valid ? cpos[k] >> 16 : 0, col = valid ? cpos[k] & 0xffff : 0;
        const int iy = ty0 + row;
        const int64_t cell = plane_base + (int64_t)row * nx + col;
        const float cur = valid ? b.src[cell] : 0.f;
        const int h = valid ? (int)t.hint[cell] : 0x44;
        const float x = fmaf((float)col, g.dx, -g.extent);
        const float y = fmaf((float)iy, g.dx, -g.extent);
        const bool captured = MODE == SL_MINTIME && hypotf(x, y) - g.radius <= 0.f;
        const float X = (float)col - center, Y = (float)iy - center;
        float best = MODE == SL_TUBE ? cur : INFINITY;
        int bu, be;
        unsigned evals = 0;
        minmax_cell(ring, pairs, make_float2(X, Y), make_float2(Y, -X),
                    (h >> 4) < 9 ? (h >> 4) : 4, (h & 15) < 9 ? (h & 15) : 4,
                    valid && !captured, best, bu, be, evals);
        evals_total += evals;
        if (valid) {
          float out;
          if (MODE == SL_TUBE) {
            out = best;
          } else {
            const float m = fminf(fmaxf(best, 0.f), 1.f);
            out = captured ? 0.f : fmaf(g.beta, m, 1.f - g.beta);
          }
          if (!isfinite(out)) bad = true;
          item_changed |= __float_as_uint(out) != __float_as_uint(cur);
          b.dst[cell] = out;
          t.hint[cell] = (uint8_t)((bu << 4) | be);
          change = fmaxf(change, fabsf(out - cur));
        }
      }
      if (ip + 1 < p1) {
        // ---- advance the ring: pair (ip+1, ip+2) replaces pair (ip-1, ip)
        cp_async_wait();
        __syncthreads();
        fill_halo();
        pair_table(ip + 1);
        __syncthreads();
        blend(ip + 2, false, false, true);
        __syncthreads();
        if (ip + 3 <= p1) load_raw(ip + 3);
        cp_async_commit();
      }
    }
    cp_async_wait();
    const int any_changed = __syncthreads_or(item_changed);
    if (tid == 0) {
      if (t.changed_out) t.changed_out[item] = any_changed ? 1u : 0u;
      atomicAdd(&b.stats->items_computed, 1ull);
    }
  }

  if (__syncthreads_or(bad) && tid == 0) atomicOr(&b.stats->nonfinite, 1u);
  for (int off = 16; off > 0; off >>= 1) {
    change = fmaxf(change, __shfl_xor_sync(0xffffffffu, change, off));
    evals_total += __shfl_xor_sync(0xffffffffu, evals_total, off);
  }
  if ((tid & 31) == 0 && evals_total) atomicAdd(&b.stats->evaluations, evals_total);
  __shared__ float warp_max[SL_TILED_MAX_THREADS / 32];
  if ((tid & 31) == 0) warp_max[tid >> 5] = change;
  __syncthreads();
  if (tid == 0) {
    float m = 0.f;
    for (int w = 0; w < (nthreads >> 5); w++) m = fmaxf(m, warp_max[w]);
    if (m > 0.f)
      atomicMax(&b.stats->residual, (unsigned long long)__double_as_longlong((double)m));
  }
}

template <int MODE>
cudaError_t launch(const SLGrid &g, const SLBackup &b, const SLTiled &t,
                   const SLTiledPlan &plan, cudaStream_t stream) {
  auto kernel = sl_tiled_kernel<MODE, kCPT>;
  cudaError_t err =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)plan.smem);
  if (err != cudaSuccess) return err;
  int device = 0, sms = 0;
  err = cudaGetDevice(&device);
  if (err != cudaSuccess) return err;
  err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (err != cudaSuccess) return err;
  int resident = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, plan.threads,
                                                      plan.smem);
  if (err != cudaSuccess) return err;
  const int64_t slots = (int64_t)sms * (resident > 0 ? resident : 1);
  const int64_t grid = plan.items < slots ? plan.items : slots;
  kernel<<<(unsigned)grid, plan.threads, plan.smem, stream>>>(g, b, t, plan);
  return cudaGetLastError();
}

}  // namespace

bool sl_tiled_plan(const SLGrid &g, int max_smem, int want_rows, SLTiledPlan *plan) {
  const int nx = g.nx;
  if (nx + 2 * kHalo > kPitch || g.nvp < 3 || g.nve < 3) return false;
  // rows per tile: about 864 cells (432 threads), at most kRowsMax rows,
  // equal tiles
  int rows = want_rows > 0 ? want_rows : 864 / nx;
  rows = rows < 1 ? 1 : (rows > kRowsMax ? kRowsMax : rows);
  const int tiles = (nx + rows - 1) / rows;
  rows = (nx + tiles - 1) / tiles;
  // two float2 heading-pair planes and one raw plane per combination, at
  // the fixed plane stride
  const size_t smem = sizeof(float) * (size_t)(5 * kCombos) * kPlane + sizeof(SLPair) * 81;
  if ((int)smem > max_smem) return false;
  const int cells = rows * nx;
  int threads = ((cells + kCPT - 1) / kCPT + 31) / 32 * 32;
  if (threads > SL_TILED_MAX_THREADS) return false;
  plan->rows = rows;
  plan->tiles_y = tiles;
  plan->psi_chunk = g.nh;
  plan->psi_chunks = 1;
  plan->threads = threads;
  plan->items = (int64_t)g.nvp * g.nve * tiles;
  plan->smem = smem;
  return true;
}

cudaError_t sl_backup_tiled(const SLGrid &g, const SLBackup &b, const SLTiled &t,
                            const SLTiledPlan &plan, cudaStream_t stream) {
  return g.mode == SL_TUBE ? launch<SL_TUBE>(g, b, t, plan, stream)
                           : launch<SL_MINTIME>(g, b, t, plan, stream);
}

}  // namespace pe
