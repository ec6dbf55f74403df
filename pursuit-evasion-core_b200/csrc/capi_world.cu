// C-ABI of the dense 8D solver handle (declared in include/pe_b200.h).
//
// Host-side restatement of the reference executable's set-up and driver
// (native_world.cpp:76-150 options, spacings, axes and dt bound; :315-336
// frame/step loop); per-cell work in world8d_exact.cu.
#include <cmath>
#include <cstring>
#include <vector>

#include "pe_internal.h"
#include "world8d.cuh"

struct pe_world {
  pe_world_params p{};
  pe::World8Grid g{};
  double dt_limit = 0;
  float *a = nullptr, *b = nullptr, *arrival = nullptr;
  float *x = nullptr, *cs = nullptr, *sn = nullptr, *pv = nullptr, *ev = nullptr;
  double *csd = nullptr, *snd = nullptr, *cdiff = nullptr, *sdiff = nullptr;
  float *p_clear = nullptr, *e_clear = nullptr;  // obstacle clearances (avoid mode 2)
  pe::World8Stats *stats = nullptr, *host_stats = nullptr;
  cudaStream_t own = nullptr, stream = nullptr;
  double t = 0;
  int64_t steps = 0;
  bool initialized = false;
  pe::LaunchTimer timer;  // launch times (profile / kernel_time)
};

namespace {

using pe::fail;

int validate(const pe_world_params *p) {
  if (!p) return fail(PE_EINVAL, "params is NULL");
  const double v[] = {p->extent, p->arena, p->capture_radius, p->p_speed_min,
                      p->p_speed_max, p->p_acceleration, p->p_curvature,
                      p->e_speed_min, p->e_speed_max, p->e_acceleration,
                      p->e_curvature, p->cfl};
  for (double x : v)
    if (!std::isfinite(x)) return fail(PE_EINVAL, "Invalid arguments: non-finite value");
  // native_world.cpp:111-117 (the arena must lie inside the grid only when
  // the square-arena avoid floor is used).
  if (p->positions < 5 || p->headings < 4 || p->p_speeds < 3 || p->e_speeds < 3 ||
      (p->avoid_mode == 1 && p->extent <= p->arena) || p->order < 1 ||
      p->order > 2 || p->cfl <= 0 || p->cfl > 1 ||
      p->p_speed_min >= p->p_speed_max || p->e_speed_min >= p->e_speed_max ||
      p->p_acceleration <= 0 || p->e_acceleration <= 0 || p->p_curvature <= 0 ||
      p->e_curvature <= 0 || p->extent <= 0 ||
      p->avoid_mode < 0 || p->avoid_mode > 2 || (p->fast != 0 && p->fast != 1))
    return fail(PE_EINVAL, "Invalid arguments");
  // each car's block of cells is indexed with 32-bit integers on the device
  const int64_t block_p = (int64_t)p->positions * p->positions * p->headings * p->p_speeds;
  const int64_t block_e = (int64_t)p->positions * p->positions * p->headings * p->e_speeds;
  if (block_p >= (int64_t)1 << 31 || block_e >= (int64_t)1 << 31)
    return fail(PE_EINVAL, "Invalid arguments: grid too large");
  return PE_OK;
}

pe::World8Grid make_grid(const pe_world_params *p) {
  pe::World8Grid g{};
  const double pi = std::acos(-1.0);
  g.n = p->positions;
  g.nh = p->headings;
  g.np = p->p_speeds;
  g.ne = p->e_speeds;
  g.order = p->order;
  g.linear_speed = p->linear_speed_boundary ? 1 : 0;
  g.avoid_mode = p->avoid_mode;
  g.extent = (float)p->extent;
  g.arena = (float)p->arena;
  g.ap = (float)p->p_acceleration;
  g.ae = (float)p->e_acceleration;
  g.kp = (float)p->p_curvature;
  g.ke = (float)p->e_curvature;
  const float dx = 2 * g.extent / (g.n - 1);
  const float dh = (float)(2 * pi / g.nh);
  const float dvp = ((float)p->p_speed_max - (float)p->p_speed_min) / (g.np - 1);
  const float dve = ((float)p->e_speed_max - (float)p->e_speed_min) / (g.ne - 1);
  const int shape[8] = {g.n, g.n, g.nh, g.np, g.n, g.n, g.nh, g.ne};
  const float spacing[8] = {dx, dx, dh, dvp, dx, dx, dh, dve};
  for (int k = 0; k < 8; k++) {
    g.shape[k] = shape[k];
    g.spacing[k] = spacing[k];
    g.inv_spacing[k] = 1.f / spacing[k];
    const float sq = spacing[k] * spacing[k];
    g.inv_spacing_sq[k] = 1.f / sq;
  }
  g.stride[7] = 1;
  for (int k = 6; k >= 0; k--) g.stride[k] = g.stride[k + 1] * shape[k + 1];
  g.cells = g.stride[0] * g.n;
  return g;
}

double dt_limit(const pe_world_params *p, const pe::World8Grid &g) {
  // native_world.cpp:133-135, in its float/double mix
  const float pabs = std::max(std::abs((float)p->p_speed_min), std::abs((float)p->p_speed_max));
  const float eabs = std::max(std::abs((float)p->e_speed_min), std::abs((float)p->e_speed_max));
  return p->cfl / (2 * double(pabs + eabs) / g.spacing[0] +
                   double(pabs * g.kp + eabs * g.ke) / g.spacing[2] +
                   double(g.ap) / g.spacing[3] + double(g.ae) / g.spacing[7]);
}

void release(pe_world *h) {
  for (void *ptr : {(void *)h->a, (void *)h->b, (void *)h->arrival, (void *)h->x,
                    (void *)h->cs, (void *)h->sn, (void *)h->pv, (void *)h->ev,
                    (void *)h->csd, (void *)h->snd, (void *)h->cdiff,
                    (void *)h->sdiff, (void *)h->stats, (void *)h->p_clear,
                    (void *)h->e_clear})
    cudaFree(ptr);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->own) cudaStreamDestroy(h->own);
}

int enter(pe_world *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->p.device));
  return PE_OK;
}

int read_stats(pe_world *h) {
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_stats, h->stats, sizeof(pe::World8Stats),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->host_stats->nonfinite)
    return fail(PE_ENONFINITE, "Nonfinite values in the signed field");
  return PE_OK;
}

int stage(pe_world *h, const float *src, float *dst, const float *base, float dt) {
  pe::World8Stage s{};
  s.src = src;
  s.dst = dst;
  s.base = base;
  s.arrival = h->arrival;
  s.x = h->x;
  s.cs = h->cs;
  s.sn = h->sn;
  s.pv = h->pv;
  s.ev = h->ev;
  s.dt = dt;
  s.tau = h->t;
  s.stats = h->stats;
  s.p_clear = h->p_clear;
  if (h->g.avoid_mode == 2 && !h->p_clear)
    return fail(PE_ESTATE, "avoid mode 2 needs pe_world_set_clearance first");
  cudaEvent_t e0 = h->timer.begin(h->stream);
  PE_CUDA_TRY(h->p.fast ? pe::world8_stage_fast(h->g, s, h->stream)
                        : pe::world8_stage(h->g, s, h->stream));
  pe::count_launches(1);
  return h->timer.end(h->stream, e0, 0);
}

int step_impl(pe_world *h, double dt) {
  PE_CUDA_TRY(cudaMemsetAsync(&h->stats->residual, 0, sizeof(unsigned long long),
                              h->stream));
  const float dtf = (float)dt;  // native_world.cpp passes Real(dt)
  int rc;
  if (h->g.order == 1) {
    rc = stage(h, h->a, h->b, nullptr, dtf);
    if (rc) return rc;
    std::swap(h->a, h->b);
  } else {
    rc = stage(h, h->a, h->b, nullptr, dtf);
    if (rc) return rc;
    rc = stage(h, h->b, h->a, h->a, dtf);
    if (rc) return rc;
  }
  h->t += dt;
  h->steps++;
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_world_cells(const pe_world_params *params, int64_t *cells) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!cells) return fail(PE_EINVAL, "cells is NULL");
  *cells = make_grid(params).cells;
  return PE_OK;
}

int pe_world_dt_limit(const pe_world_params *params, double *dt) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!dt) return fail(PE_EINVAL, "dt is NULL");
  *dt = dt_limit(params, make_grid(params));
  return PE_OK;
}

int pe_world_create(const pe_world_params *params, pe_world **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  PE_CUDA_TRY(cudaSetDevice(params->device));
  pe_world *h = new pe_world();
  h->p = *params;
  h->g = make_grid(params);
  h->dt_limit = dt_limit(params, h->g);
  const pe::World8Grid &g = h->g;
  // Axes exactly as native_world.cpp:138-150 (float), plus double trig.
  const double pi = std::acos(-1.0);
  std::vector<float> x(g.n), cs(g.nh), sn(g.nh), pv(g.np), ev(g.ne);
  std::vector<double> csd(g.nh), snd(g.nh), cdiff(g.nh * g.nh), sdiff(g.nh * g.nh);
  for (int i = 0; i < g.n; i++) x[i] = -g.extent + i * g.spacing[0];
  for (int i = 0; i < g.nh; i++) {
    const double angle = -pi + i * 2 * pi / g.nh;
    cs[i] = (float)std::cos(angle);
    sn[i] = (float)std::sin(angle);
    csd[i] = std::cos(angle);
    snd[i] = std::sin(angle);
  }
  for (int e = 0; e < g.nh; e++)
    for (int q = 0; q < g.nh; q++) {
      const double delta = (-pi + e * 2 * pi / g.nh) - (-pi + q * 2 * pi / g.nh);
      cdiff[e * g.nh + q] = std::cos(delta);
      sdiff[e * g.nh + q] = std::sin(delta);
    }
  for (int i = 0; i < g.np; i++) pv[i] = (float)params->p_speed_min + i * g.spacing[3];
  for (int i = 0; i < g.ne; i++) ev[i] = (float)params->e_speed_min + i * g.spacing[7];
  const size_t bytes = sizeof(float) * (size_t)g.cells;
  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  auto upload = [&](auto **dst, const auto &src) {
    using T = typename std::remove_reference<decltype(src[0])>::type;
    take(cudaMalloc(dst, sizeof(T) * src.size()));
    if (err == cudaSuccess)
      take(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
  };
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->a, bytes));
  take(cudaMalloc(&h->b, bytes));
  take(cudaMalloc(&h->arrival, bytes));
  take(cudaMalloc(&h->stats, sizeof(pe::World8Stats)));
  take(cudaMallocHost(&h->host_stats, sizeof(pe::World8Stats)));
  if (err == cudaSuccess) {
    upload(&h->x, x);
    upload(&h->cs, cs);
    upload(&h->sn, sn);
    upload(&h->pv, pv);
    upload(&h->ev, ev);
    upload(&h->csd, csd);
    upload(&h->snd, snd);
    upload(&h->cdiff, cdiff);
    upload(&h->sdiff, sdiff);
    take(cudaMemset(h->stats, 0, sizeof(pe::World8Stats)));
  }
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_world_create");
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_world_init_contact(pe_world *h, double p_length, double p_width,
                          double e_length, double e_width) {
  int rc = enter(h);
  if (rc) return rc;
  if (!(p_length > 0 && p_width > 0 && e_length > 0 && e_width > 0))
    return fail(PE_EINVAL, "footprint sides must be positive");
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::World8Stats), h->stream));
  PE_CUDA_TRY(pe::world8_init_contact(h->g, h->csd, h->snd, h->cdiff, h->sdiff,
                                      p_length, p_width, e_length, e_width, h->a,
                                      h->arrival, h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = 0;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_world_set_clearance(pe_world *h, const float *p_clear, const float *e_clear) {
  int rc = enter(h);
  if (rc) return rc;
  if (!p_clear || !e_clear) return fail(PE_EINVAL, "clearance arrays are NULL");
  const size_t count = (size_t)h->g.n * h->g.n * h->g.nh;
  for (size_t i = 0; i < count; i++)
    if (!std::isfinite(p_clear[i]) || !std::isfinite(e_clear[i]))
      return fail(PE_EINVAL, "non-finite clearance");
  if (!h->p_clear) PE_CUDA_TRY(cudaMalloc(&h->p_clear, sizeof(float) * count));
  if (!h->e_clear) PE_CUDA_TRY(cudaMalloc(&h->e_clear, sizeof(float) * count));
  PE_CUDA_TRY(cudaMemcpyAsync(h->p_clear, p_clear, sizeof(float) * count,
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaMemcpyAsync(h->e_clear, e_clear, sizeof(float) * count,
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_world_init_map(pe_world *h) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->p_clear) return fail(PE_ESTATE, "pe_world_set_clearance before pe_world_init_map");
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::World8Stats), h->stream));
  PE_CUDA_TRY(pe::world8_init_map(h->g, (float)h->p.capture_radius, h->p_clear, h->e_clear,
                                  h->a, h->arrival, h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = 0;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_world_init_square(pe_world *h) {
  int rc = enter(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::World8Stats), h->stream));
  PE_CUDA_TRY(pe::world8_init_square(h->g, h->x, (float)h->p.capture_radius, h->a,
                                     h->arrival, h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = 0;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_world_init_field(pe_world *h, const float *field, const float *arrival,
                        double start_time) {
  int rc = enter(h);
  if (rc) return rc;
  if (!field) return fail(PE_EINVAL, "field is NULL");
  if (!std::isfinite(start_time) || start_time < 0)
    return fail(PE_EINVAL, "start_time must be finite and >= 0");
  const size_t bytes = sizeof(float) * (size_t)h->g.cells;
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::World8Stats), h->stream));
  PE_CUDA_TRY(cudaMemcpyAsync(h->a, field, bytes, cudaMemcpyHostToDevice, h->stream));
  if (arrival) {
    PE_CUDA_TRY(cudaMemcpyAsync(h->arrival, arrival, bytes, cudaMemcpyHostToDevice,
                                h->stream));
  } else {
    PE_CUDA_TRY(pe::world8_init_arrival(h->g, h->a, h->arrival, (float)start_time,
                                        h->stream));
    pe::count_launches(1);
  }
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = start_time;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_world_advance(pe_world *h, double goal, int64_t *steps_taken) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "advance before init");
  if (!std::isfinite(goal)) return fail(PE_EINVAL, "goal must be finite");
  int64_t taken = 0;
  while (h->t < goal - 1e-10) {  // native_world.cpp:320-330
    rc = step_impl(h, std::min(h->dt_limit, goal - h->t));
    if (rc) return rc;
    taken++;
  }
  if (steps_taken) *steps_taken = taken;
  return PE_OK;
}

int pe_world_step(pe_world *h, double dt) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "step before init");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(PE_EINVAL, "dt must be > 0");
  return step_impl(h, dt);
}

int pe_world_time(const pe_world *h, double *t, int64_t *steps) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (t) *t = h->t;
  if (steps) *steps = h->steps;
  return PE_OK;
}

int pe_world_synchronize(pe_world *h) {
  int rc = enter(h);
  if (rc) return rc;
  return read_stats(h);
}

int pe_world_copy_field(pe_world *h, float *host_field) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_field) return fail(PE_EINVAL, "host_field is NULL");
  PE_CUDA_TRY(cudaMemcpyAsync(host_field, h->a, sizeof(float) * (size_t)h->g.cells,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_world_copy_arrival(pe_world *h, float *host_arrival) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_arrival) return fail(PE_EINVAL, "host_arrival is NULL");
  PE_CUDA_TRY(cudaMemcpyAsync(host_arrival, h->arrival,
                              sizeof(float) * (size_t)h->g.cells,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_world_residual(pe_world *h, double *residual) {
  int rc = enter(h);
  if (rc) return rc;
  rc = read_stats(h);
  if (rc) return rc;
  if (residual) std::memcpy(residual, &h->host_stats->residual, sizeof(double));
  return PE_OK;
}

int pe_world_set_stream(pe_world *h, void *cuda_stream) {
  int rc = enter(h);
  if (rc) return rc;
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own;
  return PE_OK;
}

int pe_world_profile(pe_world *h, int enable) {
  int rc = enter(h);
  if (rc) return rc;
  return h->timer.reset(enable != 0);
}

int pe_world_kernel_time(pe_world *h, double *total_ms, int64_t *launches) {
  int rc = enter(h);
  if (rc) return rc;
  rc = h->timer.harvest(true);
  if (rc) return rc;
  if (total_ms) *total_ms = h->timer.ms(0);
  if (launches) *launches = h->timer.launches(0);
  return PE_OK;
}

int pe_world_destroy(pe_world *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
