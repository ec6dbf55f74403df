// Relative 5D ENO/LF stage, exact variant: double local arithmetic evaluated
// in the order of the reference executable (native_relative.cpp:38-67 slopes,
// :124-172 stage), float32 storage.  This file is compiled with
// -fmad=false: no multiply-add contraction, IEEE double division, so each
// stored float equals the reference CPU's bit for bit.
//
// One thread per cell of the padded layout.  blockIdx.y enumerates (vP, vE),
// blockIdx.z the heading, and the x dimension covers the (y, x) plane, so
// that the CTAs in flight cover the speed neighbours of one heading (their
// planes stay in L2).  The kernel waits on its 21 stencil loads per cell, so
// it runs 12 CTAs of 128 threads per SM at 40 registers, spills included:
// 3.70 / 4.30 ms per stage at config 2 against 5.51 / 6.54 ms at 6 CTAs per
// SM (76-80 registers), same results.
#include "relative5d_exact.cuh"

namespace pe {
namespace {

template <int ORDER, int BLEND, typename T = float>
__global__ void __launch_bounds__(128, 12)
    rel5_stage_exact_kernel(const Rel5Grid g, const Rel5Stage s) {
  __shared__ double scratch[4];
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  double change_abs = 0, change_up = 0;
  bool bad = false;
  if (cell < g.nx * g.nx) {
    const int ix = cell % g.nx, iy = cell / g.nx;
    const int ip = blockIdx.z;
    const int ie = blockIdx.y % g.nve, iv = g.own_lo + (int)blockIdx.y / g.nve;
    const int64_t j = ((int64_t)(iv - g.slab_lo) * g.nve + ie) * g.se + (int64_t)ip * g.sp +
                      (int64_t)iy * g.sy + ix;
    exact::cell_update<ORDER, BLEND, T>(g, s, ix, iy, ip, iv, ie, j, change_abs, change_up,
                                        bad);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0)
    atomicOr(&s.stats->nonfinite, 1u);
  if (BLEND || ORDER == 1) {
    const double m_abs = exact::block_max(change_abs, scratch);
    const double m_up = exact::block_max(change_up, scratch);
    if (threadIdx.x == 0) {
      exact::atomic_max_nonneg(&s.stats->residual, m_abs);
      exact::atomic_max_nonneg(&s.stats->increase, m_up);
    }
  }
}

__global__ void rel5_broadcast_f64_kernel(const double *__restrict__ plane,
                                          double *__restrict__ field, int64_t n,
                                          int64_t plane_size) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    field[j] = plane[j % plane_size];
}

}  // namespace

cudaError_t rel5_broadcast_plane_f64(const Rel5Grid &g, const double *plane, double *field,
                                     cudaStream_t stream) {
  rel5_broadcast_f64_kernel<<<148 * 16, 256, 0, stream>>>(plane, field, g.n, g.sp);
  return cudaGetLastError();
}

cudaError_t rel5_stage_f64_storage(const Rel5Grid &g, const Rel5Stage &s, int blend,
                                   cudaStream_t stream) {
  const int threads = 128;
  const dim3 grid((g.nx * g.nx + threads - 1) / threads, g.nvp * g.nve, g.nh);
  if (g.order == 1)
    rel5_stage_exact_kernel<1, 0, double><<<grid, threads, 0, stream>>>(g, s);
  else if (blend)
    rel5_stage_exact_kernel<2, 1, double><<<grid, threads, 0, stream>>>(g, s);
  else
    rel5_stage_exact_kernel<2, 0, double><<<grid, threads, 0, stream>>>(g, s);
  return cudaGetLastError();
}

cudaError_t rel5_stage_f64(const Rel5Grid &g, const Rel5Stage &s, int blend,
                           cudaStream_t stream) {
  const int threads = 128;
  const int slabs = g.own_n > 0 ? g.own_n : g.nvp;
  const dim3 grid((g.nx * g.nx + threads - 1) / threads, slabs * g.nve, g.nh);
  if (g.order == 1)
    rel5_stage_exact_kernel<1, 0><<<grid, threads, 0, stream>>>(g, s);
  else if (blend)
    rel5_stage_exact_kernel<2, 1><<<grid, threads, 0, stream>>>(g, s);
  else
    rel5_stage_exact_kernel<2, 0><<<grid, threads, 0, stream>>>(g, s);
  return cudaGetLastError();
}

}  // namespace pe
