// Persistent batched stage loop shared by the exact and the float32 batched
// kernels (relative5d_batch_exact.cu, relative5d_batch_tiled.cu).
//
// The CTAs walk, for every RK2 step k and each of its two stages, the work
// items of the solves that still have a step k (solves are sorted by step
// count, so these are a prefix of the batch's item list), then meet at a
// grid-wide barrier before the next stage.  A work item is `rows` y rows
// of one (vP, vE, psi) plane of one solve; `Cell::update<BLEND>` is the
// per-cell arithmetic.
//
// The barrier is a counter and a generation word in global memory.  Every
// wait is bounded: after kSpinLimit polls the CTA sets the timeout flag and
// leaves; the others then time out at the same or the next barrier, so a
// launch that is not fully co-resident ends with an error instead of
// hanging.
#pragma once
#include "relative5d_batch.cuh"

namespace pe {
namespace batch_impl {

constexpr unsigned kSpinLimit = 1u << 24;  // several seconds with the back-off below

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *word, double value) {
  // non-negative doubles order like their bit patterns
  if (value > 0) atomicMax(word, (unsigned long long)__double_as_longlong(value));
}

// Block maximum of a non-negative double (blockDim.x = kRel5BatchThreads).
__device__ __forceinline__ double block_max(double v, double *scratch) {
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, scratch[w]);
  __syncthreads();
  return m;
}

__device__ __forceinline__ unsigned load_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier number `round` (1, 2, ...); false on timeout.
__device__ inline bool grid_barrier(unsigned *sync, unsigned round) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    __threadfence();
    const unsigned arrived = atomicAdd(&sync[0], 1u) + 1;
    if (arrived == round * gridDim.x) {
      __threadfence();
      atomicExch(&sync[1], round);  // release
    } else {
      unsigned spins = 0;
      while (load_acquire(&sync[1]) < round) {
        if (load_acquire(&sync[2]) != 0u || ++spins > kSpinLimit) {
          atomicOr(&sync[2], 1u);
          ok = 0;
          break;
        }
        __nanosleep(256);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ int find_solve(const Rel5BatchArgs &A, int64_t item) {
  int lo = 0, hi = A.count - 1;  // last solve with item_base <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (A.solves[mid].item_base <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// One stage of every active item.  A CTA's items (blockIdx.x, +gridDim.x,
// ...) mostly fall in the same solve as the one before, so the solve's
// descriptor is looked up (binary search) and staged in shared memory only
// when the item leaves the cached solve's range, and the residual
// reductions (block maxima, atomics) run once per solve and CTA rather
// than once per item.
template <int BLEND, class Cell>
__device__ void stage_items(const Rel5BatchArgs &A, int step, int64_t n_items,
                            double *scratch, Rel5Grid *sg) {
  int64_t lo = 0, hi = 0;  // item range of the cached solve
  const Rel5BatchSolve *S = nullptr;
  Rel5Stage s{};
  int rows = 1, blocks = 1;
  double change_abs = 0, change_up = 0;
  bool bad = false;
  auto flush = [&]() {
    if (!S) return;
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&S->stats->nonfinite, 1u);
    if (BLEND) {
      const double m_abs = block_max(change_abs, scratch);
      const double m_up = block_max(change_up, scratch);
      if (threadIdx.x == 0) {
        atomic_max_nonneg(&S->stats->residual, m_abs);
        atomic_max_nonneg(&S->stats->increase, m_up);
      }
    }
    change_abs = change_up = 0;
    bad = false;
  };
  for (int64_t item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (item < lo || item >= hi) {  // the same for every thread of the CTA
      flush();
      S = &A.solves[find_solve(A, item)];
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
      blocks = (sg->nx + rows - 1) / rows;
    }
    const Rel5Grid &g = *sg;
    int64_t local = item - lo;
    const int rb = (int)(local % blocks);
    local /= blocks;
    const int ip = (int)(local % g.nh);
    local /= g.nh;
    const int ie = (int)(local % g.nve);
    const int iv = (int)(local / g.nve);
    const int y0 = rb * rows, y1 = min(g.nx, y0 + rows);
    const int cells = (y1 - y0) * g.nx;
    const int64_t plane = (((int64_t)iv * g.nve + ie) * g.nh + ip) * g.sp;
    for (int c = threadIdx.x; c < cells; c += blockDim.x) {
      const int iy = y0 + c / g.nx, ix = c % g.nx;
      double ca = 0, cu = 0;
      Cell::template update<BLEND>(g, s, ix, iy, ip, iv, ie, plane + (int64_t)iy * g.sy + ix,
                                   ca, cu, bad);
      change_abs = fmax(change_abs, ca);
      change_up = fmax(change_up, cu);
    }
  }
  flush();
}

// 4 CTAs per SM (64 registers, spills included): the exact cell update
// waits on its stencil loads, and at its natural 146 registers only one
// CTA fits per SM (32 exact solves of seed 0: 5.73 s against 16.47 s).
template <class Cell>
__global__ void __launch_bounds__(kRel5BatchThreads, 4)
    rel5_batch_kernel(const Rel5BatchArgs A) {
  __shared__ double scratch[kRel5BatchThreads / 32];
  __shared__ Rel5Grid sg;  // grid of the solve whose items the CTA is on
  unsigned round = 0;
  for (int step = 0; step < A.max_steps; step++) {
    const int64_t n_items = A.active_items[step];
    // the residual of a solve is that of its last step: clear it once the
    // previous step is complete (the barrier before this stage)
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < A.count;
         k += gridDim.x * blockDim.x)
      if (step < A.solves[k].nsteps) A.solves[k].stats->residual = 0ull;
    stage_items<0, Cell>(A, step, n_items, scratch, &sg);
    if (!grid_barrier(A.sync, ++round)) break;
    stage_items<1, Cell>(A, step, n_items, scratch, &sg);
    if (!grid_barrier(A.sync, ++round)) break;
  }
}

template <class Cell>
int grid_size() {
  int device = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rel5_batch_kernel<Cell>,
                                                    kRel5BatchThreads, 0) != cudaSuccess)
    return 0;
  return sms * per_sm;
}

template <class Cell>
cudaError_t launch(const Rel5BatchArgs &args, int grid, cudaStream_t stream) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kRel5BatchThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, rel5_batch_kernel<Cell>, args);
}

}  // namespace batch_impl
}  // namespace pe
