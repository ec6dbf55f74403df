// Relative 5D semi-Lagrangian min-max backup, shared-memory tiled form.
//
// Same semantics as sl_backup_kernel (semilag5d.cu), restructured for
// throughput.  A persistent CTA owns a work item: one (vP, vE) speed pair,
// `rows` y rows at full x width, and a run of headings psi.  The speed
// interpolation of every successor only mixes the three vP and three vE
// slabs around the item, with weights that depend on the acceleration
// alone, so the item stages, for each of the 9 (pursuer accel, evader
// accel) combinations, the speed-blended (y, x) plane of three consecutive
// headings in a shared-memory ring (27 planes, rows + 4 by 72 floats, with
// two halo cells on every side holding the linear extension of the field
// beyond the position box).  Every (pursuer, evader) action pair is then a
// bilinear gather of 4 corners in each of two ring planes plus a heading
// lerp: 8 shared-memory loads instead of 32 global ones.
//
// The heading ring advances one plane per psi step: the raw slab rows of
// the plane after next are fetched with cp.async while the current plane
// is computed, extended into the halo, blended and stored over the plane
// that is no longer needed.
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

struct __align__(16) SLPair {  // one (pursuer, evader) action pair at the current heading
  float ox, oy;     // successor offset in local ring coordinates
  float c, s;       // the pursuer's turn: successor = R(c, s) (X, Y) + (ox, oy)
  float wp;         // heading weight of the upper plane
  unsigned lo, hi;  // ring offsets of the lower / upper heading plane, minus
                    // the magic bits of the packed (row, col) index
  float pad;
};
static_assert(sizeof(SLPair) == 32, "pair table entry is 32 bytes");

__device__ __forceinline__ int mod3(int q) {
  const int r = q % 3;
  return r < 0 ? r + 3 : r;
}

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

// Interpolated value of one action pair at a cell with centred index
// coordinates P = (X, Y) and Q = (Y, -X).  Both position axes, and the two
// heading planes, are carried side by side in packed FP32 pairs.
__device__ __forceinline__ float pair_value(const float *ring, const SLPair &p, float2 P,
                                            float2 Q) {
  const float2 F = __ffma2_rn(make_float2(p.c, p.c), P,
                              __ffma2_rn(make_float2(p.s, p.s), Q, make_float2(p.ox, p.oy)));
  const float2 T = __fadd2_rn(__fadd2_rn(F, make_float2(-0.5f, -0.5f)),
                              make_float2(kMagic, kMagic));  // round(F - 0.5) + magic
  const float2 W = __fadd2_rn(F, __fadd2_rn(make_float2(kMagic, kMagic), make_float2(-T.x, -T.y)));
  const unsigned idx = __float_as_uint(T.y) * (unsigned)kPitch + __float_as_uint(T.x);
  const float *a = ring + (int)(idx + p.lo);
  const float *b = ring + (int)(idx + p.hi);
  // (lower plane, upper plane) pairs of the four corners
  const float2 v00 = make_float2(a[0], b[0]), v01 = make_float2(a[1], b[1]);
  const float2 v10 = make_float2(a[kPitch], b[kPitch]);
  const float2 v11 = make_float2(a[kPitch + 1], b[kPitch + 1]);
  const float2 wx = make_float2(W.x, W.x), wy = make_float2(W.y, W.y);
  const float2 r0 = __ffma2_rn(wx, __fadd2_rn(v01, make_float2(-v00.x, -v00.y)), v00);
  const float2 r1 = __ffma2_rn(wx, __fadd2_rn(v11, make_float2(-v10.x, -v10.y)), v10);
  const float2 r = __ffma2_rn(wy, __fadd2_rn(r1, make_float2(-r0.x, -r0.y)), r0);
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
__device__ __forceinline__ void minmax_cell(const float *ring, const SLPair *pairs, float2 P,
                                            float2 Q, int hu, int he, bool live, float &best,
                                            int &bu, int &be) {
  bu = hu;
  be = he;
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
  const int rr = plan.rows + 2 * kHalo;  // staged rows
  const int pl = rr * kPitch;            // floats per staged plane
  float *ring = smem;                    // [combo][slot][rr][kPitch]
  float *raw = ring + 3 * kCombos * pl;  // [slab][rr][kPitch]
  SLPair *pairs = reinterpret_cast<SLPair *>(raw + kCombos * pl);

  const int nx = g.nx, nh = g.nh;
  const int tid = threadIdx.x, nthreads = blockDim.x;
  const float center = 0.5f * (float)(nx - 1);
  const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;
  float change = 0.f;
  bool bad = false;

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
    const int in_rows = gy_hi - gy_lo;

    // raw slab rows of heading plane q (unwrapped) -> raw, asynchronously;
    // one warp per (slab, row), lanes along x
    auto load_raw = [&](int q) {
      const int w = wrap_psi(q, nh);
      for (int rw = warp; rw < kCombos * in_rows; rw += nwarps) {
        const int s = rw / in_rows, gy = gy_lo + (rw - s * in_rows);
        const int va = ps.base + s / 3, vb = es.base + s % 3;
        const float *src = b.src + ((((int64_t)va * g.nve + vb) * nh + w) * nx + gy) * nx;
        float *dst = raw + s * pl + (gy - ty0 + kHalo) * kPitch + kHalo;
        for (int gx = lane; gx < nx; gx += 32) cp_async4(dst + gx, src + gx);
      }
    };
    // halo of the raw plane (needs the in-box rows in place): the two
    // columns on each side of an in-box row (one thread per slab, row and
    // column), whole rows beyond the box (lanes along x)
    auto fill_halo = [&]() {
      const int srows = trows + 2 * kHalo;
      const int side = kCombos * in_rows * 2 * kHalo;
      for (int k = tid; k < side; k += nthreads) {
        const int s = k / (in_rows * 2 * kHalo), r = k - s * (in_rows * 2 * kHalo);
        const int gy = gy_lo + r / (2 * kHalo), q = r % (2 * kHalo);
        const int gx = q < kHalo ? q - kHalo : nx + q - kHalo;
        float *plane = raw + s * pl;
        plane[(gy - ty0 + kHalo) * kPitch + gx + kHalo] = extended(plane, gx, gy, nx, ty0);
      }
      for (int rw = warp; rw < kCombos * srows; rw += nwarps) {
        const int s = rw / srows, lr = rw - s * srows;
        const int gy = ty0 - kHalo + lr;
        if (gy >= 0 && gy < nx) continue;
        float *plane = raw + s * pl;
        for (int lc = lane; lc < nx + 2 * kHalo; lc += 32)
          plane[lr * kPitch + lc] = extended(plane, lc - kHalo, gy, nx, ty0);
      }
    };
    // speed blends of the raw plane into ring slot `slot` (whole rows of the
    // pitch: the pad columns past nx + 4 hold unused values, never read)
    auto blend = [&](int slot) {
      const int count = (trows + 2 * kHalo) * kPitch;
      for (int off = tid; off < count; off += nthreads) {
        float v[9];
#pragma unroll
        for (int s = 0; s < 9; s++) v[s] = raw[s * pl + off];
        float pv[3][3];  // [pursuer accel][evader slab]
#pragma unroll
        for (int a = 0; a < 3; a++) {
          const int lo = ps.slot[a];
          const float w = ps.w[a], w0 = 1.f - w;
#pragma unroll
          for (int e = 0; e < 3; e++) {
            const float x0 = lo == 0 ? v[e] : v[3 + e];
            const float x1 = lo == 0 ? v[3 + e] : v[6 + e];
            pv[a][e] = fmaf(w, x1, w0 * x0);
          }
        }
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int e = 0; e < 3; e++) {
            const int lo = es.slot[e];
            const float w = es.w[e], w0 = 1.f - w;
            const float x0 = lo == 0 ? pv[a][0] : pv[a][1];
            const float x1 = lo == 0 ? pv[a][1] : pv[a][2];
            ring[((a * 3 + e) * 3 + slot) * pl + off] = fmaf(w, x1, w0 * x0);
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
        p.ox = fmaf(pa.c, dxp, pa.s * dyp) * g.ihx + center + (float)kHalo;
        p.oy = fmaf(pa.c, dyp, -pa.s * dxp) * g.ihx + center + (float)(kHalo - ty0);
        p.c = pa.c;
        p.s = pa.s;
        const float delta = ea.turn_idx - pa.turn_idx;
        const float fl = floorf(delta);
        p.wp = delta - fl;
        const int combo = (up / 3) * 3 + ue / 3;
        const int q = ip + (int)fl;
        const unsigned bias = kMagicBits * (unsigned)(kPitch + 1);
        p.lo = (unsigned)((combo * 3 + mod3(q)) * pl) - bias;
        p.hi = (unsigned)((combo * 3 + mod3(q + 1)) * pl) - bias;
        p.pad = 0.f;
        pairs[k] = p;
      }
    };

    // warm-up: planes p0-1, p0, p0+1 into the ring
    for (int q = p0 - 1; q <= p0 + 1; q++) {
      load_raw(q);
      cp_async_commit_wait();
      __syncthreads();
      fill_halo();
      if (q == p0 + 1) pair_table(p0);
      __syncthreads();
      blend(mod3(q));
      __syncthreads();
    }
    if (p0 + 2 <= p1) load_raw(p0 + 2);
    cp_async_commit();

    for (int ip = p0; ip < p1; ip++) {
      // ---- compute the cells of heading ip (one cell of each thread at a time)
#pragma unroll 1
      for (int k = 0; k < CPT; k++) {
        const int c = tid + k * nthreads;
        const bool valid = c < trows * nx;
        const int row = valid ? c / nx : 0, col = valid ? c - row * nx : 0;
        const int iy = ty0 + row;
        const int64_t cell = ((((int64_t)iv * g.nve + ie) * nh + ip) * nx + iy) * nx + col;
        const float cur = valid ? b.src[cell] : 0.f;
        const int h = valid ? (int)t.hint[cell] : 0x44;
        const float x = fmaf((float)col, g.dx, -g.extent);
        const float y = fmaf((float)iy, g.dx, -g.extent);
        const bool captured = MODE == SL_MINTIME && hypotf(x, y) - g.radius <= 0.f;
        const float X = (float)col - center, Y = (float)iy - center;
        float best = MODE == SL_TUBE ? cur : INFINITY;
        int bu, be;
        minmax_cell(ring, pairs, make_float2(X, Y), make_float2(Y, -X),
                    (h >> 4) < 9 ? (h >> 4) : 4, (h & 15) < 9 ? (h & 15) : 4,
                    valid && !captured, best, bu, be);
        if (valid) {
          float out;
          if (MODE == SL_TUBE) {
            out = best;
          } else {
            const float m = fminf(fmaxf(best, 0.f), 1.f);
            out = captured ? 0.f : fmaf(g.beta, m, 1.f - g.beta);
          }
          if (!isfinite(out)) bad = true;
          b.dst[cell] = out;
          t.hint[cell] = (uint8_t)((bu << 4) | be);
          change = fmaxf(change, fabsf(out - cur));
        }
      }
      if (ip + 1 < p1) {
        // ---- advance the ring: plane ip+2 replaces plane ip-1
        cp_async_wait();
        __syncthreads();
        fill_halo();
        pair_table(ip + 1);
        __syncthreads();
        blend(mod3(ip + 2));
        __syncthreads();
        if (ip + 3 <= p1) load_raw(ip + 3);
        cp_async_commit();
      }
    }
    cp_async_wait();
    __syncthreads();
  }

  if (__syncthreads_or(bad) && tid == 0) atomicOr(&b.stats->nonfinite, 1u);
  for (int off = 16; off > 0; off >>= 1)
    change = fmaxf(change, __shfl_xor_sync(0xffffffffu, change, off));
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
  // rows per tile: about 864 cells (432 threads), at most 16 rows, equal tiles
  int rows = want_rows > 0 ? want_rows : 864 / nx;
  rows = rows < 1 ? 1 : (rows > 16 ? 16 : rows);
  const int tiles = (nx + rows - 1) / rows;
  rows = (nx + tiles - 1) / tiles;
  const int rr = rows + 2 * kHalo;
  const size_t smem = sizeof(float) * (size_t)(4 * kCombos) * rr * kPitch +
                      sizeof(SLPair) * 81;
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
