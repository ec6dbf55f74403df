// C-ABI of the relative 5D solver handle (declared in include/pe_b200.h).
//
// Host-side restatement of the reference executable's driver
// (native_relative.cpp:68-90 set-up, :91-100 init, :173-190 step loop); the
// per-cell work runs in relative5d_fast.cu / relative5d_exact.cu.
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "pe_internal.h"
#include "relative5d.cuh"
#include "relative5d_host.h"

struct pe_relative {
  pe_relative_params p{};
  pe::Rel5Grid g{};
  pe::Rel5Tile tile{};
  double limit = 0;
  float *a = nullptr, *b = nullptr, *arrival = nullptr, *plane = nullptr;
  double *sn = nullptr, *cs = nullptr;
  float *snf = nullptr, *csf = nullptr;
  pe::Rel5Stats *stats = nullptr;       // device
  pe::Rel5Stats *host_stats = nullptr;  // pinned mirror
  cudaStream_t own = nullptr, stream = nullptr;
  double t = 0;
  int64_t steps = 0;
  bool initialized = false;
  pe::LaunchTimer timer;  // per-stage launch times (pe_relative_profile)
  double exit_r = 0, exit_r2 = 0;  // local exit (0: none)
  int2 *exit_keep = nullptr;        // its kept x range per y row (float32 kernels)
  // asynchronous history output: two dense snapshot buffers, filled on the
  // compute stream and copied out on their own stream
  float *snap[2] = {nullptr, nullptr};
  cudaEvent_t snap_ready[2] = {nullptr, nullptr}, snap_free[2] = {nullptr, nullptr};
  cudaStream_t copy_stream = nullptr;
};

namespace {

using pe::fail;
using pe::rel5host::cfl_limit;
using pe::rel5host::make_grid;
using pe::rel5host::validate;


void release(pe_relative *h) {
  cudaFree(h->a);
  cudaFree(h->b);
  cudaFree(h->arrival);
  cudaFree(h->plane);
  cudaFree(h->sn);
  cudaFree(h->cs);
  cudaFree(h->snf);
  cudaFree(h->csf);
  cudaFree(h->stats);
  cudaFree(h->exit_keep);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  for (int i = 0; i < 2; i++) {
    cudaFree(h->snap[i]);
    if (h->snap_ready[i]) cudaEventDestroy(h->snap_ready[i]);
    if (h->snap_free[i]) cudaEventDestroy(h->snap_free[i]);
  }
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->own) cudaStreamDestroy(h->own);
}

int launch_stage(pe_relative *h, int stage, const float *src, float *dst,
                 double dt, int blend) {
  pe::Rel5Stage s{};
  s.src = src;
  s.dst = dst;
  s.arrival = h->arrival;
  s.sn = h->sn;
  s.cs = h->cs;
  s.snf = h->snf;
  s.csf = h->csf;
  s.dt = dt;
  s.t = h->t;
  s.stats = h->stats;
  s.exit_r = h->exit_r;
  s.exit_r2 = h->exit_r2;
  s.exit_keep = h->exit_r2 > 0 ? h->exit_keep : nullptr;
  cudaEvent_t e0 = h->timer.begin(h->stream);
  const cudaError_t err =
      h->p.precision == PE_LOCAL_F64
          ? pe::rel5_stage_f64(h->g, s, blend, h->stream)
          : pe::rel5_stage_f32(h->g, h->tile, s, blend, h->stream);
  if (err != cudaSuccess) return pe::cuda_fail(err, "relative stage launch");
  pe::count_launches(1);
  return h->timer.end(h->stream, e0, stage);
}

int step_impl(pe_relative *h, double dt) {
  PE_CUDA_TRY(cudaMemsetAsync(&h->stats->residual, 0, sizeof(unsigned long long),
                              h->stream));
  int rc;
  if (h->g.order == 1) {
    rc = launch_stage(h, 0, h->a, h->b, dt, 0);
    if (rc) return rc;
    std::swap(h->a, h->b);
  } else {
    rc = launch_stage(h, 0, h->a, h->b, dt, 0);
    if (rc) return rc;
    rc = launch_stage(h, 1, h->b, h->a, dt, 1);
    if (rc) return rc;
  }
  h->t += dt;
  h->steps += 1;
  return PE_OK;
}

int read_stats(pe_relative *h) {
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_stats, h->stats, sizeof(pe::Rel5Stats),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->host_stats->timeout)
    return fail(PE_ETIMEOUT, "a bounded device wait gave up");
  if (h->host_stats->nonfinite)
    return fail(PE_ENONFINITE, "Nonfinite field update");
  return PE_OK;
}

int enter(pe_relative *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->p.device));
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_relative_cells(const pe_relative_params *params, int64_t *cells) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!cells) return fail(PE_EINVAL, "cells is NULL");
  *cells = make_grid(params).n;
  return PE_OK;
}

int pe_relative_cfl_limit(const pe_relative_params *params, double *dt_limit) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!dt_limit) return fail(PE_EINVAL, "dt_limit is NULL");
  *dt_limit = cfl_limit(params, make_grid(params));
  return PE_OK;
}

int pe_relative_create(const pe_relative_params *params, pe_relative **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  PE_CUDA_TRY(cudaSetDevice(params->device));
  pe_relative *h = new pe_relative();
  h->p = *params;
  h->g = make_grid(params);
  h->limit = cfl_limit(params, h->g);
  h->tile = pe::rel5_default_tile(h->g);
  const size_t bytes = sizeof(float) * (size_t)h->g.n_padded;
  const int nh = h->g.nh;
  std::vector<double> sn(nh), cs(nh);
  std::vector<float> snf(nh), csf(nh);
  const double pi = std::acos(-1.0);
  for (int k = 0; k < nh; k++) {
    const double q = -pi + k * h->g.dphi;  // native_relative.cpp:84-89
    sn[k] = std::sin(q);
    cs[k] = std::cos(q);
    snf[k] = (float)sn[k];
    csf[k] = (float)cs[k];
  }
  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->a, bytes));
  take(cudaMalloc(&h->b, bytes));
  take(cudaMalloc(&h->arrival, bytes));
  take(cudaMalloc(&h->plane, sizeof(float) * (size_t)h->g.sp));
  take(cudaMalloc(&h->sn, sizeof(double) * nh));
  take(cudaMalloc(&h->cs, sizeof(double) * nh));
  take(cudaMalloc(&h->snf, sizeof(float) * nh));
  take(cudaMalloc(&h->csf, sizeof(float) * nh));
  take(cudaMalloc(&h->stats, sizeof(pe::Rel5Stats)));
  take(cudaMallocHost(&h->host_stats, sizeof(pe::Rel5Stats)));
  if (err == cudaSuccess) {
    take(cudaMemcpy(h->sn, sn.data(), sizeof(double) * nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->cs, cs.data(), sizeof(double) * nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->snf, snf.data(), sizeof(float) * nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->csf, csf.data(), sizeof(float) * nh, cudaMemcpyHostToDevice));
    take(cudaMemset(h->stats, 0, sizeof(pe::Rel5Stats)));
  }
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_relative_create");
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_relative_set_stream(pe_relative *h, void *cuda_stream) {
  int rc = enter(h);
  if (rc) return rc;
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own;
  return PE_OK;
}

int pe_relative_init(pe_relative *h, const float *initial,
                     const float *arrival, double start_time) {
  int rc = enter(h);
  if (rc) return rc;
  if (!std::isfinite(start_time) || start_time < 0)
    return fail(PE_EINVAL, "start_time must be finite and >= 0");
  const size_t bytes = sizeof(float) * (size_t)h->g.n;  // dense host field
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::Rel5Stats), h->stream));
  if (!initial) {
    // The circular capture field of native_relative.cpp:91-100, one (y, x)
    // plane in double on the host, cast to float, broadcast on the device.
    const int nx = h->g.nx;
    std::vector<float> plane((size_t)nx * nx);
    for (int iy = 0; iy < nx; iy++) {
      const double y = -h->g.extent + iy * h->g.dx;
      for (int ix = 0; ix < nx; ix++)
        plane[(size_t)iy * nx + ix] = (float)(
            std::hypot(-h->g.extent + ix * h->g.dx, y) - h->p.capture_radius);
    }
    PE_CUDA_TRY(cudaMemcpyAsync(h->plane, plane.data(),
                                sizeof(float) * plane.size(),
                                cudaMemcpyHostToDevice, h->stream));
    PE_CUDA_TRY(pe::rel5_init(h->g, h->plane, h->a, h->arrival,
                              (float)start_time, h->stream));
    pe::count_launches(1);
    PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  } else {
    // Dense host field -> stage buffer -> padded field.
    PE_CUDA_TRY(cudaMemcpyAsync(h->b, initial, bytes, cudaMemcpyHostToDevice,
                                h->stream));
    PE_CUDA_TRY(pe::rel5_unpack(h->g, h->b, h->a, h->stream));
    pe::count_launches(1);
    if (arrival) {
      PE_CUDA_TRY(pe::rel5_init(h->g, nullptr, h->a, h->arrival,
                                (float)start_time, h->stream));
      PE_CUDA_TRY(cudaMemcpyAsync(h->b, arrival, bytes, cudaMemcpyHostToDevice,
                                  h->stream));
      PE_CUDA_TRY(pe::rel5_unpack(h->g, h->b, h->arrival, h->stream));
      pe::count_launches(2);
    } else {
      PE_CUDA_TRY(pe::rel5_init(h->g, nullptr, h->a, h->arrival,
                                (float)start_time, h->stream));
      pe::count_launches(1);
    }
    PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  h->t = start_time;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_relative_advance(pe_relative *h, double goal, int64_t *steps_taken) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "advance before init");
  if (!std::isfinite(goal)) return fail(PE_EINVAL, "goal must be finite");
  int64_t taken = 0;
  while (h->t < goal - 1e-12) {
    const double dt = std::min(h->limit, goal - h->t);
    rc = step_impl(h, dt);
    if (rc) return rc;
    taken++;
  }
  if (steps_taken) *steps_taken = taken;
  return PE_OK;
}

int pe_relative_step(pe_relative *h, double dt) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "step before init");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(PE_EINVAL, "dt must be > 0");
  return step_impl(h, dt);
}

int pe_relative_time(const pe_relative *h, double *t, int64_t *steps) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (t) *t = h->t;
  if (steps) *steps = h->steps;
  return PE_OK;
}

int pe_relative_synchronize(pe_relative *h) {
  int rc = enter(h);
  if (rc) return rc;
  return read_stats(h);
}

int pe_relative_init_plane(pe_relative *h, const float *plane, int64_t plane_size,
                           double start_time) {
  int rc = enter(h);
  if (rc) return rc;
  const int64_t nx2 = (int64_t)h->g.nx * h->g.nx;
  if (!plane || (plane_size != nx2 && plane_size != nx2 * h->g.nh))
    return fail(PE_EINVAL, "plane must hold positions^2 or headings * positions^2 values");
  if (!std::isfinite(start_time) || start_time < 0)
    return fail(PE_EINVAL, "start_time must be finite and >= 0");
  for (int64_t i = 0; i < plane_size; i++)
    if (!std::isfinite(plane[i])) return fail(PE_EINVAL, "non-finite plane value");
  float *dplane = nullptr;
  PE_CUDA_TRY(cudaMalloc(&dplane, sizeof(float) * (size_t)plane_size));
  cudaError_t err = cudaMemcpyAsync(dplane, plane, sizeof(float) * (size_t)plane_size,
                                    cudaMemcpyHostToDevice, h->stream);
  if (err == cudaSuccess) err = cudaMemsetAsync(h->stats, 0, sizeof(pe::Rel5Stats), h->stream);
  if (err == cudaSuccess)
    err = pe::rel5_init(h->g, dplane, h->a, h->arrival, (float)start_time, h->stream,
                        plane_size);
  if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
  cudaFree(dplane);
  if (err != cudaSuccess) return pe::cuda_fail(err, "pe_relative_init_plane");
  pe::count_launches(1);
  h->t = start_time;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_relative_set_exit(pe_relative *h, double radius, double radius_squared) {
  int rc = enter(h);
  if (rc) return rc;
  if (!std::isfinite(radius) || !std::isfinite(radius_squared) || radius < 0 ||
      radius_squared < 0 || (radius > 0) != (radius_squared > 0))
    return fail(PE_EINVAL, "exit radius must be finite and >= 0");
  if (radius > 0 && !(radius < h->g.extent))
    return fail(PE_EINVAL, "Local exit radius must lie inside the numerical grid");
  if (radius > 0) {
    if (!h->exit_keep) PE_CUDA_TRY(cudaMalloc(&h->exit_keep, sizeof(int2) * h->g.nx));
    cudaError_t err = pe::rel5_exit_rows(h->g, (float)radius_squared, h->exit_keep, h->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
    if (err != cudaSuccess) return pe::cuda_fail(err, "pe_relative_set_exit");
    pe::count_launches(1);
  }
  h->exit_r = radius;
  h->exit_r2 = radius_squared;
  return PE_OK;
}

int pe_relative_probe(pe_relative *h, int64_t n, const int64_t *indices, const double *weights,
                      double *host_out) {
  int rc = enter(h);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!indices || !weights || !host_out)))
    return fail(PE_EINVAL, "bad probe arrays");
  if (n == 0) return PE_OK;
  for (int64_t i = 0; i < 32 * n; i++)
    if (indices[i] < 0 || indices[i] >= h->g.n || !std::isfinite(weights[i]))
      return fail(PE_EINVAL, "probe stencil out of range");
  int64_t *didx = nullptr;
  double *dw = nullptr, *dout = nullptr;
  cudaError_t err = cudaMalloc(&didx, sizeof(int64_t) * 32 * (size_t)n);
  if (err == cudaSuccess) err = cudaMalloc(&dw, sizeof(double) * 32 * (size_t)n);
  if (err == cudaSuccess) err = cudaMalloc(&dout, sizeof(double) * (size_t)n);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(didx, indices, sizeof(int64_t) * 32 * (size_t)n,
                          cudaMemcpyHostToDevice, h->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(dw, weights, sizeof(double) * 32 * (size_t)n, cudaMemcpyHostToDevice,
                          h->stream);
  if (err == cudaSuccess) err = pe::rel5_probe(h->g, h->a, n, didx, dw, dout, h->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(host_out, dout, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                          h->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
  cudaFree(didx);
  cudaFree(dw);
  cudaFree(dout);
  if (err != cudaSuccess) return pe::cuda_fail(err, "pe_relative_probe");
  pe::count_launches(1);
  return PE_OK;
}

int pe_relative_snapshot(pe_relative *h, int32_t slot) {
  int rc = enter(h);
  if (rc) return rc;
  if (slot < 0 || slot > 1) return fail(PE_EINVAL, "snapshot slot must be 0 or 1");
  if (!h->initialized) return fail(PE_ESTATE, "snapshot before init");
  if (!h->copy_stream) {
    PE_CUDA_TRY(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; i++) {
      PE_CUDA_TRY(cudaMalloc(&h->snap[i], sizeof(float) * (size_t)h->g.n));
      PE_CUDA_TRY(cudaEventCreateWithFlags(&h->snap_ready[i], cudaEventDisableTiming));
      PE_CUDA_TRY(cudaEventCreateWithFlags(&h->snap_free[i], cudaEventDisableTiming));
      PE_CUDA_TRY(cudaEventRecord(h->snap_free[i], h->copy_stream));
    }
  }
  // the previous copy out of this slot must be done before it is refilled
  PE_CUDA_TRY(cudaStreamWaitEvent(h->stream, h->snap_free[slot], 0));
  PE_CUDA_TRY(pe::rel5_pack(h->g, h->a, h->snap[slot], h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaEventRecord(h->snap_ready[slot], h->stream));
  return PE_OK;
}

int pe_relative_copy_snapshot(pe_relative *h, int32_t slot, float *host_field) {
  int rc = enter(h);
  if (rc) return rc;
  if (slot < 0 || slot > 1 || !host_field) return fail(PE_EINVAL, "bad slot or NULL buffer");
  if (!h->copy_stream) return fail(PE_ESTATE, "no snapshot taken");
  PE_CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->snap_ready[slot], 0));
  PE_CUDA_TRY(cudaMemcpyAsync(host_field, h->snap[slot], sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToHost, h->copy_stream));
  PE_CUDA_TRY(cudaEventRecord(h->snap_free[slot], h->copy_stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->copy_stream));
  return PE_OK;
}

int pe_host_alloc(size_t bytes, void **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  PE_CUDA_TRY(cudaHostAlloc(out, bytes, cudaHostAllocDefault));
  return PE_OK;
}

int pe_host_free(void *ptr) {
  if (ptr) PE_CUDA_TRY(cudaFreeHost(ptr));
  return PE_OK;
}

int pe_relative_copy_field(pe_relative *h, float *host_field) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_field) return fail(PE_EINVAL, "host_field is NULL");
  // Padded field -> dense stage buffer -> host (the stage buffer is free
  // between steps).
  PE_CUDA_TRY(pe::rel5_pack(h->g, h->a, h->b, h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaMemcpyAsync(host_field, h->b, sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_relative_copy_arrival(pe_relative *h, float *host_arrival) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_arrival) return fail(PE_EINVAL, "host_arrival is NULL");
  PE_CUDA_TRY(pe::rel5_pack(h->g, h->arrival, h->b, h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaMemcpyAsync(host_arrival, h->b, sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_relative_device_field(pe_relative *h, float **device_field) {
  if (!h || !device_field) return fail(PE_EINVAL, "NULL argument");
  *device_field = h->a;
  return PE_OK;
}

int pe_relative_row_pitch(const pe_relative *h, int32_t *floats) {
  if (!h || !floats) return fail(PE_EINVAL, "NULL argument");
  *floats = h->g.xp;
  return PE_OK;
}

int pe_relative_set_tile(pe_relative *h, int32_t rows, int32_t psi_chunk) {
  int rc = enter(h);
  if (rc) return rc;
  pe::Rel5Tile t{rows, psi_chunk};
  if (rows == 0 && psi_chunk == 0) t = pe::rel5_default_tile(h->g);
  if (!pe::rel5_tile_valid(h->g, t))
    return fail(PE_EINVAL, "tile rows=%d psi_chunk=%d does not fit this grid",
                rows, psi_chunk);
  h->tile = t;
  return PE_OK;
}

int pe_relative_get_tile(const pe_relative *h, int32_t *rows,
                         int32_t *psi_chunk) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (rows) *rows = h->tile.rows;
  if (psi_chunk) *psi_chunk = h->tile.psi_chunk;
  return PE_OK;
}

int pe_relative_kernel_info(const pe_relative *h, int32_t *threads,
                            int32_t *smem_bytes, int32_t *resident_ctas) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  const int consumer_warps = (h->tile.rows * (h->g.xp / 4) + 31) / 32;
  if (threads) *threads = 32 * (consumer_warps + 1);
  if (smem_bytes) *smem_bytes = (int32_t)pe::rel5_fast_smem_bytes(h->g, h->tile);
  if (resident_ctas) *resident_ctas = pe::rel5_last_resident_ctas();
  return PE_OK;
}

int pe_relative_stats(pe_relative *h, double *residual, double *max_increase) {
  int rc = enter(h);
  if (rc) return rc;
  rc = read_stats(h);
  if (rc) return rc;
  double r, inc;
  std::memcpy(&r, &h->host_stats->residual, sizeof r);
  std::memcpy(&inc, &h->host_stats->increase, sizeof inc);
  if (residual) *residual = r;
  if (max_increase) *max_increase = inc;
  return PE_OK;
}

int pe_relative_profile(pe_relative *h, int enable) {
  int rc = enter(h);
  if (rc) return rc;
  return h->timer.reset(enable != 0);
}

int pe_relative_kernel_time(pe_relative *h, int stage, double *total_ms,
                            int64_t *launches) {
  int rc = enter(h);
  if (rc) return rc;
  if (stage != 0 && stage != 1) return fail(PE_EINVAL, "stage must be 0 or 1");
  rc = h->timer.harvest(true);
  if (rc) return rc;
  if (total_ms) *total_ms = h->timer.ms(stage);
  if (launches) *launches = h->timer.launches(stage);
  return PE_OK;
}

int pe_relative_destroy(pe_relative *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
