// Compact eight-state semi-Lagrangian contact game: capture field, fused
// min-max backup and product-stencil queries, for the dense pair layout and
// the pair-packed domain (src/pursuit_evasion/local_game/grid_game.py,
// local_game/reference.py:122-134).
//
// Backup.  The reference runs, per chunk of 256 pursuer states and per
// pursuer action u, one launch that interpolates the pursuer successor of
// every (ip, ie') pair into a temporary [chunk][n_e] array and one launch
// that reduces over the evader replies (grid_game.py:286-333, :384-421), and
// in the packed memory-saving mode copies every output tile to the host.
// Here one persistent launch does the whole backup: a CTA takes a pursuer
// state ip, and for each allowed u builds the interpolated row
//   g[ie'] = sum_k wp[ip,u,k] V(idp[ip,u,k], ie')
// in shared memory (coalesced reads of 16 field rows), then every thread
// reduces its cells (ip, ie) over the evader replies with 16 shared-memory
// gathers per reply, keeping the running minimum over u in the output
// array.  The reference's early exit (a reply at least as bad as the best
// value so far drops the action) is kept, so the values equal the
// reference's.  Rows longer than the shared-memory budget go to a
// per-CTA scratch row in global memory (L2-resident).
#include <algorithm>
#include <cmath>
#include <map>
#include <utility>
#include <vector>

#include "pe_internal.h"

namespace pe {
namespace {

constexpr int kThreads = 512;
constexpr int kStencil = 16;
constexpr int kMaxRowBytes = 192 * 1024;

struct CompactDev {
  int np, ne, npa, nea;
  // reach lists: for each pursuer position class, the evader states within
  // the exit radius plus the evader stencil reach (the only entries of an
  // interpolated row that a reduction reads)
  const int *p_class;        // [np] position class of each pursuer state
  const int *reach_index;    // concatenated evader ids
  const long long *reach_start;  // [classes + 1]
  const float4 *p_pose, *e_pose;
  const int *p_ids, *e_ids;
  const float *p_w, *e_w;
  const uint8_t *p_allowed, *e_allowed;
  // pair-packed domain
  const int *p_position, *lookup, *e_indices, *counts;
  const long long *offsets;
  int positions, max_count;
  float exit_value;  // exit radius
  float reach;       // exit radius + evader stencil reach (packed rows)
};

// Oriented-rectangle separating-axis value of two footprints in float32
// (geometry.py:15-36 as evaluated by the reference's CUDA initializer,
// grid_game.py:193-201): the largest of the gaps along both bodies' axes.
__device__ __forceinline__ float contact_value(float4 a, float4 b, float pl, float pw,
                                               float el, float ew) {
  const float dx = b.x - a.x, dy = b.y - a.y;
  const float rel = b.z - a.z;
  const float ca = fabsf(cosf(rel)), sa = fabsf(sinf(rel));
  const float cp = cosf(a.z), sp = sinf(a.z), ce = cosf(b.z), se = sinf(b.z);
  // gaps along the pursuer's axes, then along the evader's
  const float gpx = fabsf(dx * cp + dy * sp) - .5f * (pl + el * ca + ew * sa);
  const float gpy = fabsf(-dx * sp + dy * cp) - .5f * (pw + el * sa + ew * ca);
  const float gex = fabsf(dx * ce + dy * se) - .5f * (el + pl * ca + pw * sa);
  const float gey = fabsf(-dx * se + dy * ce) - .5f * (ew + pl * sa + pw * ca);
  return fmaxf(fmaxf(gpx, gpy), fmaxf(gex, gey));
}

__global__ void init_dense_kernel(CompactDev d, float *f, float pl, float pw, float el,
                                  float ew) {
  const long long n = (long long)d.np * d.ne;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const int ip = (int)(j / d.ne), ie = (int)(j - (long long)ip * d.ne);
    const float4 a = d.p_pose[ip], b = d.e_pose[ie];
    const float dx = b.x - a.x, dy = b.y - a.y;
    f[j] = dx * dx + dy * dy > d.exit_value * d.exit_value
               ? d.exit_value
               : contact_value(a, b, pl, pw, el, ew);
  }
}

__global__ void init_packed_kernel(CompactDev d, float *f, float pl, float pw, float el,
                                   float ew) {
  for (int ip = blockIdx.x; ip < d.np; ip += gridDim.x) {
    const int pos = d.p_position[ip];
    const int count = d.counts[pos];
    const float4 a = d.p_pose[ip];
    for (int k = threadIdx.x; k < count; k += blockDim.x) {
      const int ie = d.e_indices[(long long)pos * d.max_count + k];
      f[d.offsets[ip] + k] = contact_value(a, d.e_pose[ie], pl, pw, el, ew);
    }
  }
}

// Value of the pursuer successor vertex `nxt` paired with evader state ie
// in the packed layout (grid_game.py:403-411).
__device__ __forceinline__ float packed_at(const CompactDev &d, const float *__restrict__ f,
                                           int nxt, int ie) {
  const int rank = __ldg(d.lookup + (long long)__ldg(d.p_position + nxt) * d.ne + ie);
  return rank < 0 ? d.exit_value : __ldg(f + __ldg(d.offsets + nxt) + rank);
}

template <bool PACKED, bool SMEM>
__global__ void __launch_bounds__(kThreads)
    backup_kernel(const CompactDev d, const float *__restrict__ cur, float *__restrict__ out,
                  float *__restrict__ scratch) {
  extern __shared__ float row_smem[];
  __shared__ long long s_row[kStencil], s_off[kStencil];
  __shared__ float s_w[kStencil];
  float *g = SMEM ? row_smem : scratch + (size_t)blockIdx.x * d.ne;
  const int tid = threadIdx.x;
  const float r2 = d.exit_value * d.exit_value;

  for (int ip = blockIdx.x; ip < d.np; ip += gridDim.x) {
    int count, pos = 0;
    long long base;
    if (PACKED) {
      pos = d.p_position[ip];
      count = d.counts[pos];
      base = d.offsets[ip];
    } else {
      count = d.ne;
      base = (long long)ip * d.ne;
    }
    const int *cell_e = PACKED ? d.e_indices + (long long)pos * d.max_count : nullptr;
    const float4 pp = d.p_pose[ip];
    const int cls = d.p_class[ip];
    const long long r_begin = d.reach_start[cls], r_end = d.reach_start[cls + 1];
    // the running minimum starts at the current value; every cell is owned
    // by the same thread for the whole pose
    for (int k = tid; k < count; k += kThreads) out[base + k] = cur[base + k];

    for (int u = 0; u < d.npa; u++) {
      if (!d.p_allowed[(long long)ip * d.npa + u]) continue;
      __syncthreads();  // the previous row's readers are done
      if (tid < kStencil) {
        const long long s = ((long long)ip * d.npa + u) * kStencil + tid;
        const int nxt = d.p_ids[s];
        const float w = d.p_w[s];
        s_w[tid] = w;
        // row bases of the vertex: its lookup row and field row (packed), its
        // field row (dense); unused vertices get 0
        if (PACKED) {
          s_row[tid] = w > 0.f ? (long long)d.p_position[nxt] * d.ne : 0;
          s_off[tid] = w > 0.f ? d.offsets[nxt] : 0;
        } else {
          s_off[tid] = w > 0.f ? (long long)nxt * d.ne : 0;
        }
      }
      __syncthreads();
      // interpolated pursuer successor against the evader states within
      // reach (entries beyond it are never read: every evader stencil vertex
      // of a cell in the exit radius lies within the reach)
      for (long long t = r_begin + tid; t < r_end; t += kThreads) {
        const int ie = __ldg(d.reach_index + t);
        float v = 0.f;
        if (PACKED) {
#pragma unroll
          for (int k = 0; k < kStencil; k++)
            if (s_w[k] > 0.f) {
              const int rank = __ldg(d.lookup + s_row[k] + ie);
              v = fmaf(s_w[k], rank < 0 ? d.exit_value : __ldg(cur + s_off[k] + rank), v);
            }
        } else {
#pragma unroll
          for (int k = 0; k < kStencil; k++)
            if (s_w[k] > 0.f) v = fmaf(s_w[k], __ldg(cur + s_off[k] + ie), v);
        }
        g[ie] = v;
      }
      __syncthreads();
      // evader replies: max with early exit against the running minimum
      for (int k = tid; k < count; k += kThreads) {
        const int ie = PACKED ? cell_e[k] : k;
        if (!PACKED) {
          const float4 ep = d.e_pose[ie];
          const float dx = pp.x - ep.x, dy = pp.y - ep.y;
          if (dx * dx + dy * dy > r2) continue;  // outside the local game
        }
        const float best = out[base + k];
        float worst = -1e30f;
        bool dropped = false;
        // the next allowed reply's stencil is loaded while this one reduces
        const uint8_t *allowed = d.e_allowed + (long long)ie * d.nea;
        int a = 0;
        while (a < d.nea && !__ldg(allowed + a)) a++;
        int4 ci[kStencil / 4];
        float4 cw[kStencil / 4];
        if (a < d.nea) {
          const long long s = ((long long)ie * d.nea + a) * kStencil;
#pragma unroll
          for (int q = 0; q < kStencil / 4; q++) {
            ci[q] = __ldg(reinterpret_cast<const int4 *>(d.e_ids + s) + q);
            cw[q] = __ldg(reinterpret_cast<const float4 *>(d.e_w + s) + q);
          }
        }
        while (a < d.nea) {
          int next = a + 1;
          while (next < d.nea && !__ldg(allowed + next)) next++;
          int4 ni[kStencil / 4];
          float4 nw[kStencil / 4];
          if (next < d.nea) {
            const long long s = ((long long)ie * d.nea + next) * kStencil;
#pragma unroll
            for (int q = 0; q < kStencil / 4; q++) {
              ni[q] = __ldg(reinterpret_cast<const int4 *>(d.e_ids + s) + q);
              nw[q] = __ldg(reinterpret_cast<const float4 *>(d.e_w + s) + q);
            }
          }
          float value = 0.f;
#pragma unroll
          for (int q = 0; q < kStencil / 4; q++) {
            if (cw[q].x > 0.f) value = fmaf(cw[q].x, g[ci[q].x], value);
            if (cw[q].y > 0.f) value = fmaf(cw[q].y, g[ci[q].y], value);
            if (cw[q].z > 0.f) value = fmaf(cw[q].z, g[ci[q].z], value);
            if (cw[q].w > 0.f) value = fmaf(cw[q].w, g[ci[q].w], value);
          }
          worst = fmaxf(worst, value);
          if (worst >= best) {
            dropped = true;
            break;
          }
          a = next;
#pragma unroll
          for (int q = 0; q < kStencil / 4; q++) {
            ci[q] = ni[q];
            cw[q] = nw[q];
          }
        }
        if (!dropped) out[base + k] = fminf(best, worst);
      }
    }
    __syncthreads();  // g and s_ids are reused by the next pose
  }
}

// Backup with every pursuer action at once (up to kMaxActions actions,
// evader state ids below 2^16): for a pursuer state the CTA builds the
// interpolated rows of all its allowed actions over the evader states within
// reach, G[u][t] for reach entry t, plus a map from evader state to t; each
// thread then walks the replies of its cells once, loading every evader
// stencil a single time and applying it to all actions still alive.  An
// action drops out once its running reply maximum reaches the cell's
// current value (it cannot lower the minimum), so the value equals the
// reference's action-by-action loop with its early exit.
constexpr int kMaxActions = 9;

template <bool PACKED>
__global__ void __launch_bounds__(kThreads)
    backup_all_kernel(const CompactDev d, const float *__restrict__ cur,
                      float *__restrict__ out, int rcap, int group) {
  extern __shared__ __align__(16) float smem[];
  float *G = smem;                                                      // [group][rcap]
  unsigned short *lmap = reinterpret_cast<unsigned short *>(G + group * rcap);  // [ne]
  __shared__ long long s_row[kMaxActions][kStencil], s_off[kMaxActions][kStencil];
  __shared__ float s_w[kMaxActions][kStencil];
  __shared__ unsigned s_allowed;
  const int tid = threadIdx.x;
  const float r2 = d.exit_value * d.exit_value;

  for (int ip = blockIdx.x; ip < d.np; ip += gridDim.x) {
    int count, pos = 0;
    long long base;
    if (PACKED) {
      pos = d.p_position[ip];
      count = d.counts[pos];
      base = d.offsets[ip];
    } else {
      count = d.ne;
      base = (long long)ip * d.ne;
    }
    const int *cell_e = PACKED ? d.e_indices + (long long)pos * d.max_count : nullptr;
    const float4 pp = d.p_pose[ip];
    const int cls = d.p_class[ip];
    const long long r_begin = d.reach_start[cls];
    const int r_n = (int)(d.reach_start[cls + 1] - r_begin);
    if (tid < d.npa * kStencil) {
      const int u = tid / kStencil, k = tid % kStencil;
      const long long s = ((long long)ip * d.npa + u) * kStencil + k;
      const bool allowed = d.p_allowed[(long long)ip * d.npa + u] != 0;
      const int nxt = d.p_ids[s];
      const float w = allowed ? d.p_w[s] : 0.f;
      s_w[u][k] = w;
      if (PACKED) {
        s_row[u][k] = w > 0.f ? (long long)d.p_position[nxt] * d.ne : 0;
        s_off[u][k] = w > 0.f ? d.offsets[nxt] : 0;
      } else {
        s_off[u][k] = w > 0.f ? (long long)nxt * d.ne : 0;
      }
    }
    if (tid == 0) {
      unsigned m = 0;
      for (int u = 0; u < d.npa; u++) m |= d.p_allowed[(long long)ip * d.npa + u] ? 1u << u : 0u;
      s_allowed = m;
    }
    __syncthreads();
    const unsigned allowed_u = s_allowed;
    for (int t = tid; t < r_n; t += kThreads)
      lmap[__ldg(d.reach_index + r_begin + t)] = (unsigned short)t;
    bool first = true;  // no group has written this pursuer state's cells yet
    for (int u0 = 0; u0 < d.npa; u0 += group) {
      const unsigned in_group = allowed_u & (((1u << group) - 1u) << u0);
      if (!in_group) continue;  // the same for the whole CTA
      // rows of the group's allowed actions over the reach list, two reach
      // entries (t, t + kThreads) per thread at a time so that the
      // dependent (lookup, field) loads of both are in flight together; the
      // second entry of an odd tail repeats the first and is not stored
      for (int t = tid; t < r_n; t += 2 * kThreads) {
        const int t2 = t + kThreads;
        const bool two = t2 < r_n;
        const int ie = __ldg(d.reach_index + r_begin + t);
        const int ie2 = two ? __ldg(d.reach_index + r_begin + t2) : ie;
        for (int u = u0; u < u0 + group && u < d.npa; u++) {
          if (!((in_group >> u) & 1u)) continue;
          float v = 0.f, v2 = 0.f;
#pragma unroll
          for (int k = 0; k < kStencil; k++) {
            // a zero-weight tap has row and offset 0, so its loads stay in
            // bounds and need no branch; only its FMA is skipped
            const float wk = s_w[u][k];
            float x, x2;
            if (PACKED) {
              const int rank = __ldg(d.lookup + s_row[u][k] + ie);
              const int rank2 = __ldg(d.lookup + s_row[u][k] + ie2);
              x = rank < 0 ? d.exit_value : __ldg(cur + s_off[u][k] + rank);
              x2 = rank2 < 0 ? d.exit_value : __ldg(cur + s_off[u][k] + rank2);
            } else {
              x = __ldg(cur + s_off[u][k] + ie);
              x2 = __ldg(cur + s_off[u][k] + ie2);
            }
            v = wk > 0.f ? fmaf(wk, x, v) : v;
            v2 = wk > 0.f ? fmaf(wk, x2, v2) : v2;
          }
          G[(u - u0) * rcap + t] = v;
          if (two) G[(u - u0) * rcap + t2] = v2;
        }
      }
      __syncthreads();
      for (int k = tid; k < count; k += kThreads) {
        const int ie = PACKED ? cell_e[k] : k;
        // the running minimum: the current value before the first group
        const float best = first ? cur[base + k] : out[base + k];
        if (!PACKED) {
          const float4 ep = d.e_pose[ie];
          const float dx = pp.x - ep.x, dy = pp.y - ep.y;
          if (dx * dx + dy * dy > r2) {  // outside the local game
            out[base + k] = best;
            continue;
          }
        }
        float worst[kMaxActions];
#pragma unroll
        for (int u = 0; u < kMaxActions; u++) worst[u] = -1e30f;
        unsigned alive = in_group >> u0;  // bit g: action u0 + g
        const uint8_t *allowed_e = d.e_allowed + (long long)ie * d.nea;
        // the stencil of reply a + 1 (and its allowed flag) is loaded while
        // reply a is reduced, so that its L2 latency overlaps the gathers;
        // a disallowed reply's stencil is loaded and dropped
        const long long s0 = (long long)ie * d.nea * kStencil;
        int4 next_i[kStencil / 4];
        float4 next_w[kStencil / 4];
        bool next_ok = false;
        if (d.nea > 0) {
          next_ok = __ldg(allowed_e) != 0;
#pragma unroll
          for (int q = 0; q < kStencil / 4; q++) {
            next_i[q] = __ldg(reinterpret_cast<const int4 *>(d.e_ids + s0) + q);
            next_w[q] = __ldg(reinterpret_cast<const float4 *>(d.e_w + s0) + q);
          }
        }
        for (int a = 0; a < d.nea && alive; a++) {
          int4 cur_i[kStencil / 4];
          float4 cur_w[kStencil / 4];
          const bool ok = next_ok;
#pragma unroll
          for (int q = 0; q < kStencil / 4; q++) {
            cur_i[q] = next_i[q];
            cur_w[q] = next_w[q];
          }
          if (a + 1 < d.nea) {
            const long long s = s0 + (long long)(a + 1) * kStencil;
            next_ok = __ldg(allowed_e + a + 1) != 0;
#pragma unroll
            for (int q = 0; q < kStencil / 4; q++) {
              next_i[q] = __ldg(reinterpret_cast<const int4 *>(d.e_ids + s) + q);
              next_w[q] = __ldg(reinterpret_cast<const float4 *>(d.e_w + s) + q);
            }
          }
          if (!ok) continue;
          int t[kStencil];
          float w[kStencil];
#pragma unroll
          for (int q = 0; q < kStencil / 4; q++) {
            const int4 i4 = cur_i[q];
            const float4 w4 = cur_w[q];
            w[4 * q] = w4.x;
            w[4 * q + 1] = w4.y;
            w[4 * q + 2] = w4.z;
            w[4 * q + 3] = w4.w;
            t[4 * q] = w4.x > 0.f ? lmap[i4.x] : 0;
            t[4 * q + 1] = w4.y > 0.f ? lmap[i4.y] : 0;
            t[4 * q + 2] = w4.z > 0.f ? lmap[i4.z] : 0;
            t[4 * q + 3] = w4.w > 0.f ? lmap[i4.w] : 0;
          }
#pragma unroll
          for (int g = 0; g < kMaxActions; g++) {
            if (!((alive >> g) & 1u)) continue;
            const float *row = G + g * rcap;
            float value = 0.f;
#pragma unroll
            for (int q = 0; q < kStencil; q++)
              value = w[q] > 0.f ? fmaf(w[q], row[t[q]], value) : value;  // t[q] = 0 at w = 0
            worst[g] = fmaxf(worst[g], value);
            if (worst[g] >= best) alive &= ~(1u << g);
          }
        }
        float result = best;
#pragma unroll
        for (int g = 0; g < kMaxActions; g++)
          if ((alive >> g) & 1u) result = fminf(result, worst[g]);
        out[base + k] = result;
      }
      __syncthreads();  // the rows are rebuilt for the next group
      first = false;
    }
    if (!allowed_u)  // no allowed action: every cell keeps its value
      for (int k = tid; k < count; k += kThreads) out[base + k] = cur[base + k];
    __syncthreads();  // the map is rebuilt for the next pursuer state
  }
}

template <bool PACKED>
__global__ void query_kernel(CompactDev d, const float *__restrict__ f, int n,
                             const int *__restrict__ pi, const float *__restrict__ pw,
                             const int *__restrict__ ei, const float *__restrict__ ew,
                             float *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float total = 0.f;
  for (int a = 0; a < kStencil; a++) {
    const float wa = pw[kStencil * i + a];
    if (!(wa > 0.f)) continue;
    const int p = pi[kStencil * i + a];
    float value = 0.f;
    for (int b = 0; b < kStencil; b++) {
      const float wb = ew[kStencil * i + b];
      if (!(wb > 0.f)) continue;
      const int e = ei[kStencil * i + b];
      const float x = PACKED ? packed_at(d, f, p, e) : f[(long long)p * d.ne + e];
      value = fmaf(wb, x, value);
    }
    total = fmaf(wa, value, total);
  }
  out[i] = total;
}

template <typename T>
int upload(const T *host, size_t count, T **dev) {
  *dev = nullptr;
  if (count == 0) return PE_OK;
  PE_CUDA_TRY(cudaMalloc(dev, count * sizeof(T)));
  PE_CUDA_TRY(cudaMemcpy(*dev, host, count * sizeof(T), cudaMemcpyHostToDevice));
  return PE_OK;
}

}  // namespace
}  // namespace pe

struct pe_compact {
  int device = 0;
  bool packed = false;
  pe::CompactDev d{};
  int64_t cells = 0;
  std::vector<void *> owned;  // device arrays of the grids and the domain
  float *field = nullptr, *next = nullptr, *scratch = nullptr;
  int grid = 0;
  size_t smem = 0;
  bool smem_row = true;
  bool all_actions = false;  // backup_all_kernel applies
  int rcap = 0;              // longest reach list
  int group = 0;             // pursuer actions per pass of backup_all_kernel
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool initialized = false;
  pe::LaunchTimer timer;
};

namespace {

using pe::fail;

int check_grid(const pe_vehicle_grid *g, const char *role) {
  if (!g || !g->pose || !g->ids || !g->weights || !g->allowed)
    return fail(PE_EINVAL, "%s grid: NULL array", role);
  if (g->states < 1 || g->actions < 1 || g->actions > 64)
    return fail(PE_EINVAL, "%s grid: %d states, %d actions", role, g->states, g->actions);
  const size_t n = (size_t)g->states * g->actions * pe::kStencil;
  for (size_t i = 0; i < n; i++) {
    const float w = g->weights[i];
    if (!std::isfinite(w)) return fail(PE_EINVAL, "%s grid: non-finite weight", role);
    if (w > 0 && (g->ids[i] < 0 || g->ids[i] >= g->states))
      return fail(PE_EINVAL, "%s grid: vertex id %d out of range", role, g->ids[i]);
  }
  for (size_t i = 0; i < (size_t)g->states * 4; i++)
    if (!std::isfinite(g->pose[i])) return fail(PE_EINVAL, "%s grid: non-finite state", role);
  return PE_OK;
}

int check_domain(const pe_pair_domain *dm, int np, int ne) {
  if (!dm->p_position || !dm->lookup || !dm->e_indices || !dm->counts || !dm->offsets)
    return fail(PE_EINVAL, "pair domain: NULL array");
  if (dm->positions < 1 || dm->max_count < 0 || dm->max_count > ne)
    return fail(PE_EINVAL, "pair domain: %d positions, %d max count", dm->positions,
                dm->max_count);
  for (int i = 0; i < dm->positions; i++) {
    const int c = dm->counts[i];
    if (c < 0 || c > dm->max_count) return fail(PE_EINVAL, "pair domain: bad count");
    for (int k = 0; k < c; k++) {
      const int ie = dm->e_indices[(size_t)i * dm->max_count + k];
      if (ie < 0 || ie >= ne || dm->lookup[(size_t)i * ne + ie] != k)
        return fail(PE_EINVAL, "pair domain: e_indices and lookup disagree");
    }
    for (int ie = 0; ie < ne; ie++) {
      const int r = dm->lookup[(size_t)i * ne + ie];
      if (r < -1 || r >= c) return fail(PE_EINVAL, "pair domain: lookup rank out of range");
    }
  }
  if (dm->offsets[0] != 0) return fail(PE_EINVAL, "pair domain: offsets[0] != 0");
  for (int ip = 0; ip < np; ip++) {
    const int pos = dm->p_position[ip];
    if (pos < 0 || pos >= dm->positions)
      return fail(PE_EINVAL, "pair domain: p_position out of range");
    if (dm->offsets[ip + 1] - dm->offsets[ip] != dm->counts[pos])
      return fail(PE_EINVAL, "pair domain: offsets disagree with counts");
  }
  return PE_OK;
}

// Position classes of the pursuer states (equal (x, y)) and, per class, the
// evader states within `reach` of it, in increasing order.
void reach_lists(const pe_vehicle_grid *p, const pe_vehicle_grid *e, double reach,
                 std::vector<int> *p_class, std::vector<int> *index,
                 std::vector<long long> *start) {
  std::map<std::pair<float, float>, int> classes;
  std::vector<std::pair<float, float>> centre;
  p_class->resize(p->states);
  for (int i = 0; i < p->states; i++) {
    const std::pair<float, float> xy(p->pose[4 * i], p->pose[4 * i + 1]);
    auto it = classes.find(xy);
    if (it == classes.end()) {
      it = classes.emplace(xy, (int)centre.size()).first;
      centre.push_back(xy);
    }
    (*p_class)[i] = it->second;
  }
  start->assign(1, 0);
  index->clear();
  // a little beyond the float32 reach test of the reference kernels, so that
  // every entry they could read is present
  const double r2 = (reach + 1e-5) * (reach + 1e-5);
  for (const auto &c : centre) {
    for (int j = 0; j < e->states; j++) {
      const double dx = (double)c.first - e->pose[4 * j];
      const double dy = (double)c.second - e->pose[4 * j + 1];
      if (dx * dx + dy * dy <= r2) index->push_back(j);
    }
    start->push_back((long long)index->size());
  }
}

// Largest centre displacement of an evader interpolation vertex with a
// positive weight, plus 1e-4 (grid_game.py:456-466).
double evader_reach(const pe_vehicle_grid *e) {
  double reach = 0;
  const size_t rows = (size_t)e->states * e->actions;
  for (size_t r = 0; r < rows; r++) {
    const size_t state = r / e->actions;
    for (int q = 0; q < pe::kStencil; q++) {
      const size_t s = r * pe::kStencil + q;
      if (!(e->weights[s] > 0)) continue;
      const int v = e->ids[s];
      const double dx = (double)e->pose[4 * v] - e->pose[4 * state];
      const double dy = (double)e->pose[4 * v + 1] - e->pose[4 * state + 1];
      reach = std::fmax(reach, std::sqrt(dx * dx + dy * dy));
    }
  }
  return reach + 1e-4;
}

void release(pe_compact *h) {
  cudaSetDevice(h->device);
  for (void *p : h->owned) cudaFree(p);
  cudaFree(h->field);
  cudaFree(h->next);
  cudaFree(h->scratch);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

template <typename T>
int own(pe_compact *h, const T *host, size_t count, const T **dev) {
  T *p = nullptr;
  const int rc = pe::upload(host, count, &p);
  if (p) h->owned.push_back(p);
  *dev = p;
  return rc;
}

int upload_grid(pe_compact *h, const pe_vehicle_grid *g, const float4 **pose,
                const int **ids, const float **w, const uint8_t **allowed) {
  const size_t n = g->states, rows = n * g->actions;
  const float *pose_f = nullptr;
  int rc = own(h, g->pose, n * 4, &pose_f);
  if (rc) return rc;
  *pose = reinterpret_cast<const float4 *>(pose_f);
  if ((rc = own(h, g->ids, rows * pe::kStencil, ids))) return rc;
  if ((rc = own(h, g->weights, rows * pe::kStencil, w))) return rc;
  return own(h, g->allowed, rows, allowed);
}

int configure_launch(pe_compact *h, int rcap) {
  int sms = 0;
  PE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  int max_smem = 0;
  PE_CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                     h->device));
  // groups of actions at once: rows of `group` actions over the longest
  // reach list and a 16-bit map of the evader states
  const size_t map_bytes = sizeof(unsigned short) * (size_t)h->d.ne + 16;
  const int64_t fit = rcap > 0 ? ((int64_t)max_smem - 4096 - (int64_t)map_bytes) /
                                     ((int64_t)sizeof(float) * rcap)
                               : 0;
  const int group = (int)std::min<int64_t>(std::min(h->d.npa, pe::kMaxActions), fit);
  const size_t all_smem = sizeof(float) * (size_t)std::max(group, 1) * rcap + map_bytes;
  if (h->d.npa <= pe::kMaxActions && h->d.ne <= 65536 && group >= 2) {
    const void *kernel = h->packed ? (const void *)pe::backup_all_kernel<true>
                                   : (const void *)pe::backup_all_kernel<false>;
    PE_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)all_smem));
    int resident = 0;
    PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, pe::kThreads,
                                                              all_smem));
    if (resident >= 1) {
      h->all_actions = true;
      h->rcap = rcap;
      h->group = group;
      h->smem = all_smem;
      const int64_t slots = (int64_t)sms * resident;
      h->grid = (int)(h->d.np < slots ? h->d.np : slots);
      return PE_OK;
    }
  }
  const size_t row = (size_t)h->d.ne * sizeof(float);
  h->smem_row = row <= (size_t)pe::kMaxRowBytes;
  h->smem = h->smem_row ? row : 0;
  const void *kernel =
      h->packed ? (h->smem_row ? (const void *)pe::backup_kernel<true, true>
                               : (const void *)pe::backup_kernel<true, false>)
                : (h->smem_row ? (const void *)pe::backup_kernel<false, true>
                               : (const void *)pe::backup_kernel<false, false>);
  PE_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)h->smem));
  int resident = 0;
  PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, pe::kThreads,
                                                            h->smem));
  if (resident < 1) return fail(PE_EINVAL, "compact backup: no resident CTA fits");
  const int64_t slots = (int64_t)sms * resident;
  h->grid = (int)(h->d.np < slots ? h->d.np : slots);
  if (!h->smem_row)
    PE_CUDA_TRY(cudaMalloc(&h->scratch, (size_t)h->grid * row));
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_compact_create(const pe_vehicle_grid *p, const pe_vehicle_grid *e,
                      const pe_pair_domain *domain, double exit_radius, int32_t device,
                      pe_compact **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = check_grid(p, "pursuer");
  if (rc) return rc;
  if ((rc = check_grid(e, "evader"))) return rc;
  if (!std::isfinite(exit_radius) || exit_radius <= 0)
    return fail(PE_EINVAL, "exit radius must be positive");
  if ((int64_t)p->states * e->states >= ((int64_t)1 << 40))
    return fail(PE_EINVAL, "pair space too large");
  if (domain && (rc = check_domain(domain, p->states, e->states))) return rc;
  int count = 0;
  PE_CUDA_TRY(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(PE_EINVAL, "no CUDA device %d", device);
  PE_CUDA_TRY(cudaSetDevice(device));

  pe_compact *h = new pe_compact;
  h->device = device;
  h->packed = domain != nullptr;
  pe::CompactDev &d = h->d;
  int rcap = 0;
  d.np = p->states;
  d.ne = e->states;
  d.npa = p->actions;
  d.nea = e->actions;
  d.exit_value = (float)exit_radius;
  d.reach = (float)(exit_radius + evader_reach(e));
  rc = upload_grid(h, p, &d.p_pose, &d.p_ids, &d.p_w, &d.p_allowed);
  if (!rc) rc = upload_grid(h, e, &d.e_pose, &d.e_ids, &d.e_w, &d.e_allowed);
  if (!rc) {
    std::vector<int> p_class, index;
    std::vector<long long> start;
    reach_lists(p, e, d.reach, &p_class, &index, &start);
    for (size_t c = 0; c + 1 < start.size(); c++)
      rcap = std::max(rcap, (int)(start[c + 1] - start[c]));
    rc = own(h, p_class.data(), p_class.size(), &d.p_class);
    if (!rc) rc = own(h, index.data(), index.size(), &d.reach_index);
    if (!rc) rc = own(h, start.data(), start.size(), &d.reach_start);
  }
  if (!rc && domain) {
    d.positions = domain->positions;
    d.max_count = domain->max_count;
    rc = own(h, domain->p_position, (size_t)d.np, &d.p_position);
    if (!rc) rc = own(h, domain->lookup, (size_t)d.positions * d.ne, &d.lookup);
    if (!rc) rc = own(h, domain->e_indices, (size_t)d.positions * d.max_count, &d.e_indices);
    if (!rc) rc = own(h, domain->counts, (size_t)d.positions, &d.counts);
    if (!rc)
      rc = own(h, reinterpret_cast<const long long *>(domain->offsets), (size_t)d.np + 1,
               &d.offsets);
    h->cells = domain->offsets[d.np];
  } else {
    h->cells = (int64_t)d.np * d.ne;
  }
  if (!rc && h->cells > 0) {
    const cudaError_t err1 = cudaMalloc(&h->field, (size_t)h->cells * sizeof(float));
    const cudaError_t err2 =
        err1 == cudaSuccess ? cudaMalloc(&h->next, (size_t)h->cells * sizeof(float)) : err1;
    if (err2 != cudaSuccess) rc = pe::cuda_fail(err2, "compact field");
  }
  if (!rc) rc = configure_launch(h, rcap);
  if (!rc) {
    const cudaError_t err = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) rc = pe::cuda_fail(err, "cudaStreamCreate");
    h->own_stream = err == cudaSuccess;
  }
  if (rc) {
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_compact_cells(const pe_compact *h, int64_t *out) {
  if (!h || !out) return fail(PE_EINVAL, "NULL argument");
  *out = h->cells;
  return PE_OK;
}

int pe_compact_init(pe_compact *h, double p_length, double p_width, double e_length,
                    double e_width) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  const double dims[4] = {p_length, p_width, e_length, e_width};
  for (double v : dims)
    if (!std::isfinite(v) || v <= 0) return fail(PE_EINVAL, "footprints must be positive");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  if (h->cells > 0) {
    if (h->packed)
      pe::init_packed_kernel<<<148 * 8, 256, 0, h->stream>>>(
          h->d, h->field, (float)p_length, (float)p_width, (float)e_length, (float)e_width);
    else
      pe::init_dense_kernel<<<148 * 8, 256, 0, h->stream>>>(
          h->d, h->field, (float)p_length, (float)p_width, (float)e_length, (float)e_width);
    PE_CUDA_TRY(cudaGetLastError());
    pe::count_launches(1);
  }
  h->initialized = true;
  return PE_OK;
}

int pe_compact_set_field(pe_compact *h, const float *host, int64_t n) {
  if (!h || !host) return fail(PE_EINVAL, "NULL argument");
  if (n != h->cells) return fail(PE_EINVAL, "field has %lld values, expected %lld",
                                 (long long)n, (long long)h->cells);
  for (int64_t i = 0; i < n; i++)
    if (!std::isfinite(host[i])) return fail(PE_EINVAL, "non-finite field value");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  PE_CUDA_TRY(cudaMemcpyAsync(h->field, host, (size_t)n * sizeof(float),
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->initialized = true;
  return PE_OK;
}

int pe_compact_backup(pe_compact *h, int32_t count) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (count < 0) return fail(PE_EINVAL, "negative backup count");
  if (!h->initialized) return fail(PE_ESTATE, "backup before init");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  for (int32_t i = 0; i < count && h->cells > 0; i++) {
    cudaEvent_t t0 = h->timer.begin(h->stream);
    if (h->all_actions) {
      if (h->packed)
        pe::backup_all_kernel<true><<<h->grid, pe::kThreads, h->smem, h->stream>>>(
            h->d, h->field, h->next, h->rcap, h->group);
      else
        pe::backup_all_kernel<false><<<h->grid, pe::kThreads, h->smem, h->stream>>>(
            h->d, h->field, h->next, h->rcap, h->group);
    } else if (h->packed) {
      if (h->smem_row)
        pe::backup_kernel<true, true><<<h->grid, pe::kThreads, h->smem, h->stream>>>(
            h->d, h->field, h->next, h->scratch);
      else
        pe::backup_kernel<true, false><<<h->grid, pe::kThreads, 0, h->stream>>>(
            h->d, h->field, h->next, h->scratch);
    } else {
      if (h->smem_row)
        pe::backup_kernel<false, true><<<h->grid, pe::kThreads, h->smem, h->stream>>>(
            h->d, h->field, h->next, h->scratch);
      else
        pe::backup_kernel<false, false><<<h->grid, pe::kThreads, 0, h->stream>>>(
            h->d, h->field, h->next, h->scratch);
    }
    PE_CUDA_TRY(cudaGetLastError());
    pe::count_launches(1);
    const int rc = h->timer.end(h->stream, t0, 0);
    if (rc) return rc;
    std::swap(h->field, h->next);
  }
  return PE_OK;
}

int pe_compact_copy_field(pe_compact *h, float *host, int64_t n) {
  if (!h || !host) return fail(PE_EINVAL, "NULL argument");
  if (n != h->cells) return fail(PE_EINVAL, "buffer has %lld values, expected %lld",
                                 (long long)n, (long long)h->cells);
  PE_CUDA_TRY(cudaSetDevice(h->device));
  PE_CUDA_TRY(cudaMemcpyAsync(host, h->field, (size_t)n * sizeof(float),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_compact_field_device(pe_compact *h, void **out) {
  if (!h || !out) return fail(PE_EINVAL, "NULL argument");
  *out = h->field;
  return PE_OK;
}

int pe_compact_query(pe_compact *h, int32_t n, const int32_t *p_ids,
                     const float *p_weights, const int32_t *e_ids, const float *e_weights,
                     float *host_out) {
  if (!h || !p_ids || !p_weights || !e_ids || !e_weights || !host_out)
    return fail(PE_EINVAL, "NULL argument");
  if (n < 0) return fail(PE_EINVAL, "negative query count");
  if (n == 0) return PE_OK;
  const size_t m = (size_t)n * pe::kStencil;
  for (size_t i = 0; i < m; i++) {
    if (p_weights[i] > 0 && (p_ids[i] < 0 || p_ids[i] >= h->d.np))
      return fail(PE_EINVAL, "query: pursuer vertex out of range");
    if (e_weights[i] > 0 && (e_ids[i] < 0 || e_ids[i] >= h->d.ne))
      return fail(PE_EINVAL, "query: evader vertex out of range");
  }
  PE_CUDA_TRY(cudaSetDevice(h->device));
  int32_t *pi = nullptr, *ei = nullptr;
  float *pw = nullptr, *ew = nullptr, *out = nullptr;
  int rc = pe::upload(p_ids, m, &pi);
  if (!rc) rc = pe::upload(p_weights, m, &pw);
  if (!rc) rc = pe::upload(e_ids, m, &ei);
  if (!rc) rc = pe::upload(e_weights, m, &ew);
  if (!rc) {
    const cudaError_t err = cudaMalloc(&out, (size_t)n * sizeof(float));
    if (err != cudaSuccess) rc = pe::cuda_fail(err, "query output");
  }
  if (!rc) {
    const int blocks = (n + 255) / 256;
    if (h->packed)
      pe::query_kernel<true><<<blocks, 256, 0, h->stream>>>(h->d, h->field, n, pi, pw, ei,
                                                            ew, out);
    else
      pe::query_kernel<false><<<blocks, 256, 0, h->stream>>>(h->d, h->field, n, pi, pw, ei,
                                                             ew, out);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
      pe::count_launches(1);
      err = cudaMemcpyAsync(host_out, out, (size_t)n * sizeof(float),
                            cudaMemcpyDeviceToHost, h->stream);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
    if (err != cudaSuccess) rc = pe::cuda_fail(err, "compact query");
  }
  cudaFree(pi);
  cudaFree(pw);
  cudaFree(ei);
  cudaFree(ew);
  cudaFree(out);
  return rc;
}

int pe_compact_set_stream(pe_compact *h, void *cuda_stream) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->own_stream) PE_CUDA_TRY(cudaStreamDestroy(h->stream));
  h->stream = static_cast<cudaStream_t>(cuda_stream);
  h->own_stream = false;
  return PE_OK;
}

int pe_compact_synchronize(pe_compact *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_compact_profile(pe_compact *h, int32_t enable) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  return h->timer.reset(enable != 0);
}

int pe_compact_kernel_time(pe_compact *h, double *ms, int64_t *launches) {
  if (!h || !ms || !launches) return fail(PE_EINVAL, "NULL argument");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  const int rc = h->timer.harvest(true);
  if (rc) return rc;
  *ms = h->timer.ms(0);
  *launches = h->timer.launches(0);
  return PE_OK;
}

int pe_compact_destroy(pe_compact *h) {
  if (!h) return PE_OK;
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
