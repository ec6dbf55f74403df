// C-ABI of the FP64-storage relative solve (declared in include/pe_b200.h):
// the exact ENO/LF stage with double values, i.e. the FP64 oracle of the CPU
// restatement (po_rel_stage_f64, itself native_relative.cpp:38-172 with
// double storage) run on the GPU so that it can reach the horizon of the
// 89M-cell table.  It measures the error of float32-storage tables; the
// reference itself stores float32 only.
//
// Dense layout [vP, vE, psi, y, x] (no row padding), two double fields, the
// heading tables and the reduction words.  The initial field is
// hypot(x, y) - r in double, computed on the host (the same libm call as
// the oracle) and broadcast on the device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pe_internal.h"
#include "relative5d.cuh"
#include "relative5d_host.h"

struct pe_relative_f64 {
  pe_relative_params p{};
  pe::Rel5Grid g{};
  double limit = 0;
  double *a = nullptr, *b = nullptr, *plane = nullptr;
  double *sn = nullptr, *cs = nullptr;
  pe::Rel5Stats *stats = nullptr;
  cudaStream_t own = nullptr, stream = nullptr;
  double t = 0;
  int64_t steps = 0;
  bool initialized = false;
};

namespace {

using pe::fail;

void release(pe_relative_f64 *h) {
  cudaFree(h->a);
  cudaFree(h->b);
  cudaFree(h->plane);
  cudaFree(h->sn);
  cudaFree(h->cs);
  cudaFree(h->stats);
  if (h->own) cudaStreamDestroy(h->own);
}

int enter(pe_relative_f64 *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->p.device));
  return PE_OK;
}

int step_impl(pe_relative_f64 *h, double dt) {
  // the residual is the last step's; the non-finite flag stays set
  PE_CUDA_TRY(cudaMemsetAsync(&h->stats->residual, 0, sizeof(unsigned long long), h->stream));
  pe::Rel5Stage s{};
  s.sn = h->sn;
  s.cs = h->cs;
  s.dt = dt;
  s.t = h->t;
  s.stats = h->stats;
  if (h->g.order == 1) {
    s.src64 = h->a;
    s.dst64 = h->b;
    PE_CUDA_TRY(pe::rel5_stage_f64_storage(h->g, s, 0, h->stream));
    std::swap(h->a, h->b);
    pe::count_launches(1);
  } else {
    s.src64 = h->a;
    s.dst64 = h->b;
    PE_CUDA_TRY(pe::rel5_stage_f64_storage(h->g, s, 0, h->stream));
    s.src64 = h->b;
    s.dst64 = h->a;
    PE_CUDA_TRY(pe::rel5_stage_f64_storage(h->g, s, 1, h->stream));
    pe::count_launches(2);
  }
  h->t += dt;
  h->steps += 1;
  return PE_OK;
}

int read_stats(pe_relative_f64 *h, pe::Rel5Stats *out) {
  PE_CUDA_TRY(cudaMemcpyAsync(out, h->stats, sizeof *out, cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (out->nonfinite) return fail(PE_ENONFINITE, "Nonfinite field update");
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_relative_f64_create(const pe_relative_params *params, pe_relative_f64 **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = pe::rel5host::validate(params);
  if (rc) return rc;
  PE_CUDA_TRY(cudaSetDevice(params->device));
  pe_relative_f64 *h = new pe_relative_f64();
  h->p = *params;
  h->g = pe::rel5host::make_grid(params);
  h->limit = pe::rel5host::cfl_limit(params, h->g);
  // dense strides: the exact stage addresses cells through them
  h->g.xp = h->g.nx;
  h->g.sy = h->g.nx;
  h->g.sp = (int64_t)h->g.nx * h->g.nx;
  h->g.se = h->g.sp * h->g.nh;
  h->g.sv = h->g.se * h->g.nve;
  h->g.n_padded = h->g.n;
  std::vector<double> sn, cs;
  pe::rel5host::heading_tables(h->g, &sn, &cs);
  const size_t bytes = sizeof(double) * (size_t)h->g.n;
  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->a, bytes));
  take(cudaMalloc(&h->b, bytes));
  take(cudaMalloc(&h->plane, sizeof(double) * (size_t)h->g.sp));
  take(cudaMalloc(&h->sn, sizeof(double) * h->g.nh));
  take(cudaMalloc(&h->cs, sizeof(double) * h->g.nh));
  take(cudaMalloc(&h->stats, sizeof(pe::Rel5Stats)));
  if (err == cudaSuccess) {
    take(cudaMemcpy(h->sn, sn.data(), sizeof(double) * h->g.nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->cs, cs.data(), sizeof(double) * h->g.nh, cudaMemcpyHostToDevice));
  }
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_relative_f64_create");
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_relative_f64_destroy(pe_relative_f64 *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return PE_OK;
}

int pe_relative_f64_set_stream(pe_relative_f64 *h, void *cuda_stream) {
  int rc = enter(h);
  if (rc) return rc;
  h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own;
  return PE_OK;
}

int pe_relative_f64_initialize(pe_relative_f64 *h) {
  int rc = enter(h);
  if (rc) return rc;
  const pe::Rel5Grid &g = h->g;
  std::vector<double> plane((size_t)g.sp);
  for (int iy = 0; iy < g.nx; iy++) {
    const double y = -g.extent + iy * g.dx;
    for (int ix = 0; ix < g.nx; ix++)
      plane[(size_t)iy * g.nx + ix] =
          std::hypot(-g.extent + ix * g.dx, y) - h->p.capture_radius;
  }
  PE_CUDA_TRY(cudaMemcpyAsync(h->plane, plane.data(), sizeof(double) * plane.size(),
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::Rel5Stats), h->stream));
  PE_CUDA_TRY(pe::rel5_broadcast_plane_f64(g, h->plane, h->a, h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));  // `plane` leaves scope
  h->t = 0;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_relative_f64_step(pe_relative_f64 *h, double dt) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "step before init");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(PE_EINVAL, "dt must be > 0");
  return step_impl(h, dt);
}

int pe_relative_f64_advance(pe_relative_f64 *h, double goal, int64_t *steps_taken) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "advance before init");
  if (!std::isfinite(goal)) return fail(PE_EINVAL, "goal must be finite");
  int64_t taken = 0;
  while (h->t < goal - 1e-12) {
    rc = step_impl(h, std::min(h->limit, goal - h->t));
    if (rc) return rc;
    taken++;
  }
  if (steps_taken) *steps_taken = taken;
  return PE_OK;
}

int pe_relative_f64_time(const pe_relative_f64 *h, double *t, int64_t *steps,
                         double *cfl_dt_limit) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (t) *t = h->t;
  if (steps) *steps = h->steps;
  if (cfl_dt_limit) *cfl_dt_limit = h->limit;
  return PE_OK;
}

int pe_relative_f64_stats(pe_relative_f64 *h, double *residual) {
  int rc = enter(h);
  if (rc) return rc;
  pe::Rel5Stats host{};
  rc = read_stats(h, &host);
  if (rc) return rc;
  if (residual) std::memcpy(residual, &host.residual, sizeof(double));
  return PE_OK;
}

int pe_relative_f64_copy_field(pe_relative_f64 *h, double *host_dst) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_dst) return fail(PE_EINVAL, "host_dst is NULL");
  if (!h->initialized) return fail(PE_ESTATE, "copy before init");
  PE_CUDA_TRY(cudaMemcpyAsync(host_dst, h->a, sizeof(double) * (size_t)h->g.n,
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  pe::Rel5Stats host{};
  return read_stats(h, &host);
}

}  // extern "C"
