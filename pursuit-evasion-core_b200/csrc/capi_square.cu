// C ABI of the legacy six-dimensional square game: the executable
// src/pursuit_evasion/dp/native_square.cpp (run by dp/native.py:14-106) as a
// GPU handle.  Options, surfaces, dt bound, frame loop and the float32 stage
// are the reference's; the stage runs in square6d_exact.cu.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pe_internal.h"
#include "square6d.cuh"

struct pe_square {
  pe_square_params p{};
  pe::Square6Grid g{};
  double dt_limit = 0;
  float *a = nullptr, *b = nullptr, *arrival = nullptr;
  float *x = nullptr, *cs = nullptr, *sn = nullptr;
  pe::Square6Stats *stats = nullptr, *host_stats = nullptr;
  cudaStream_t own = nullptr, stream = nullptr;
  double t = 0;
  int64_t steps = 0;
  bool initialized = false;
  pe::LaunchTimer timer;
};

namespace {

using pe::fail;

int validate(const pe_square_params *p) {
  if (!p) return fail(PE_EINVAL, "params is NULL");
  const double v[] = {p->extent,  p->arena,       p->capture_radius, p->p_speed,
                      p->e_speed, p->p_turn_rate, p->e_turn_rate,    p->cfl};
  for (double x : v)
    if (!std::isfinite(x)) return fail(PE_EINVAL, "Invalid arguments: non-finite value");
  // native_square.cpp:81-84, plus the model's positive speeds and turn rates
  if (p->positions < 5 || p->headings < 4 || p->extent <= p->arena || p->order < 1 ||
      p->order > 2 || p->cfl <= 0 || p->cfl > 1 || p->arena <= 0 ||
      p->capture_radius <= 0 || p->p_speed <= 0 || p->e_speed <= 0 ||
      p->p_turn_rate <= 0 || p->e_turn_rate <= 0)
    return fail(PE_EINVAL, "Invalid grid/configuration/output");
  const int64_t block = (int64_t)p->positions * p->positions * p->headings;
  if (block >= ((int64_t)1 << 31)) return fail(PE_EINVAL, "grid too large");
  return PE_OK;
}

pe::Square6Grid make_grid(const pe_square_params *p) {
  pe::Square6Grid g{};
  g.n = p->positions;
  g.nh = p->headings;
  g.order = p->order;
  const double pi = std::acos(-1.0);
  const float extent = (float)p->extent;
  g.dx = 2 * extent / (g.n - 1);  // native_square.cpp:87
  g.dh = (float)(2 * pi / g.nh);
  {
    const float dx2 = g.dx * g.dx, dh2 = g.dh * g.dh;  // rounded as the stage forms them
    g.rdx = 1.f / g.dx;
    g.rdx2 = 1.f / dx2;
    g.rdh = 1.f / g.dh;
    g.rdh2 = 1.f / dh2;
  }
  g.vp = (float)p->p_speed;
  g.ve = (float)p->e_speed;
  g.wp = (float)p->p_turn_rate;
  g.we = (float)p->e_turn_rate;
  g.arena = (float)p->arena;
  const int shape[6] = {g.n, g.n, g.nh, g.n, g.n, g.nh};
  g.stride[5] = 1;
  for (int k = 4; k >= 0; k--) g.stride[k] = g.stride[k + 1] * shape[k + 1];
  g.cells = g.stride[0] * g.n;
  return g;
}

// native_square.cpp:94-95 in its float/double mix.
double dt_limit(const pe_square_params *p, const pe::Square6Grid &g) {
  const float vp = (float)p->p_speed, ve = (float)p->e_speed;
  const float wp = (float)p->p_turn_rate, we = (float)p->e_turn_rate;
  return p->cfl / (2 * (vp + ve) / double(g.dx) + (wp + we) / double(g.dh));
}

void release(pe_square *h) {
  for (void *ptr : {(void *)h->a, (void *)h->b, (void *)h->arrival, (void *)h->x,
                    (void *)h->cs, (void *)h->sn, (void *)h->stats})
    cudaFree(ptr);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->own) cudaStreamDestroy(h->own);
}

int enter(pe_square *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->p.device));
  return PE_OK;
}

int read_stats(pe_square *h) {
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_stats, h->stats, sizeof(pe::Square6Stats),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->host_stats->nonfinite) return fail(PE_ENONFINITE, "Nonfinite field update");
  return PE_OK;
}

int stage(pe_square *h, const float *src, float *dst, const float *base, float dt) {
  pe::Square6Stage s{};
  s.src = src;
  s.dst = dst;
  s.base = base;
  s.arrival = h->arrival;
  s.x = h->x;
  s.cs = h->cs;
  s.sn = h->sn;
  s.dt = dt;
  s.tau = h->t;
  s.stats = h->stats;
  cudaEvent_t e0 = h->timer.begin(h->stream);
  PE_CUDA_TRY(pe::square6_stage(h->g, s, h->stream));
  pe::count_launches(1);
  return h->timer.end(h->stream, e0, 0);
}

int step_impl(pe_square *h, double dt) {
  PE_CUDA_TRY(cudaMemsetAsync(&h->stats->residual, 0, sizeof(unsigned long long), h->stream));
  const float dtf = (float)dt;  // native_square.cpp:189 passes Real(dt)
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

int pe_square_cells(const pe_square_params *params, int64_t *cells) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!cells) return fail(PE_EINVAL, "cells is NULL");
  *cells = make_grid(params).cells;
  return PE_OK;
}

int pe_square_dt_limit(const pe_square_params *params, double *dt) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!dt) return fail(PE_EINVAL, "dt is NULL");
  *dt = dt_limit(params, make_grid(params));
  return PE_OK;
}

int pe_square_create(const pe_square_params *params, pe_square **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  int count = 0;
  PE_CUDA_TRY(cudaGetDeviceCount(&count));
  if (params->device < 0 || params->device >= count)
    return fail(PE_EINVAL, "no CUDA device %d", params->device);
  PE_CUDA_TRY(cudaSetDevice(params->device));
  pe_square *h = new pe_square();
  h->p = *params;
  h->g = make_grid(params);
  h->dt_limit = dt_limit(params, h->g);
  const pe::Square6Grid &g = h->g;
  // axes exactly as native_square.cpp:98-104 (float)
  const double pi = std::acos(-1.0);
  const float extent = (float)params->extent;
  std::vector<float> x(g.n), cs(g.nh), sn(g.nh);
  for (int i = 0; i < g.n; i++) x[i] = -extent + i * g.dx;
  for (int i = 0; i < g.nh; i++) {
    cs[i] = (float)std::cos(-pi + i * 2 * pi / g.nh);
    sn[i] = (float)std::sin(-pi + i * 2 * pi / g.nh);
  }
  const size_t bytes = sizeof(float) * (size_t)g.cells;
  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  auto upload = [&](float **dst, const std::vector<float> &src) {
    take(cudaMalloc(dst, sizeof(float) * src.size()));
    if (err == cudaSuccess)
      take(cudaMemcpy(*dst, src.data(), sizeof(float) * src.size(), cudaMemcpyHostToDevice));
  };
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->a, bytes));
  take(cudaMalloc(&h->b, bytes));
  take(cudaMalloc(&h->arrival, bytes));
  take(cudaMalloc(&h->stats, sizeof(pe::Square6Stats)));
  take(cudaMallocHost(&h->host_stats, sizeof(pe::Square6Stats)));
  if (err == cudaSuccess) {
    upload(&h->x, x);
    upload(&h->cs, cs);
    upload(&h->sn, sn);
    take(cudaMemset(h->stats, 0, sizeof(pe::Square6Stats)));
  }
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_square_create");
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_square_init(pe_square *h) {
  int rc = enter(h);
  if (rc) return rc;
  // Surfaces of native_square.cpp:110-128 on the host (the same libm hypotf
  // as the reference executable), one value per (xP, yP, xE, yE).
  const pe::Square6Grid &g = h->g;
  const float extent = (float)h->p.extent, L = (float)h->p.arena,
              r = (float)h->p.capture_radius;
  std::vector<float> x(g.n);
  for (int i = 0; i < g.n; i++) x[i] = -extent + i * g.dx;
  std::vector<float> block((size_t)g.n * g.n * g.n * g.n);
  size_t k = 0;
  for (int xp = 0; xp < g.n; xp++)
    for (int yp = 0; yp < g.n; yp++)
      for (int xe = 0; xe < g.n; xe++)
        for (int ye = 0; ye < g.n; ye++) {
          const float target = std::min(std::hypot(x[xp] - x[xe], x[yp] - x[ye]) - r,
                                        L - std::max(std::abs(x[xe]), std::abs(x[ye])));
          const float avoid = std::max(std::abs(x[xp]), std::abs(x[yp])) - L + 1e-6f;
          block[k++] = std::max(target, avoid);
        }
  float *dblock = nullptr;
  PE_CUDA_TRY(cudaMalloc(&dblock, sizeof(float) * block.size()));
  cudaError_t err = cudaMemcpyAsync(dblock, block.data(), sizeof(float) * block.size(),
                                    cudaMemcpyHostToDevice, h->stream);
  if (err == cudaSuccess) err = pe::square6_init(g, dblock, h->a, h->arrival, h->stream);
  if (err == cudaSuccess) err = cudaMemsetAsync(h->stats, 0, sizeof(pe::Square6Stats), h->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
  cudaFree(dblock);
  if (err != cudaSuccess) return pe::cuda_fail(err, "pe_square_init");
  pe::count_launches(1);
  h->t = 0;
  h->steps = 0;
  h->initialized = true;
  return PE_OK;
}

int pe_square_advance(pe_square *h, double goal, int64_t *steps_taken) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "advance before init");
  if (!std::isfinite(goal)) return fail(PE_EINVAL, "goal must be finite");
  int64_t taken = 0;
  while (h->t < goal - 1e-10) {  // native_square.cpp:186-198
    rc = step_impl(h, std::min(h->dt_limit, goal - h->t));
    if (rc) return rc;
    taken++;
  }
  if (steps_taken) *steps_taken = taken;
  return PE_OK;
}

int pe_square_time(const pe_square *h, double *t, int64_t *steps) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (t) *t = h->t;
  if (steps) *steps = h->steps;
  return PE_OK;
}

int pe_square_synchronize(pe_square *h) {
  int rc = enter(h);
  if (rc) return rc;
  return read_stats(h);
}

int pe_square_copy_field(pe_square *h, float *host_field) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_field) return fail(PE_EINVAL, "host_field is NULL");
  PE_CUDA_TRY(cudaMemcpyAsync(host_field, h->a, sizeof(float) * (size_t)h->g.cells,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_square_copy_arrival(pe_square *h, float *host_arrival) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_arrival) return fail(PE_EINVAL, "host_arrival is NULL");
  PE_CUDA_TRY(cudaMemcpyAsync(host_arrival, h->arrival, sizeof(float) * (size_t)h->g.cells,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_square_residual(pe_square *h, double *residual) {
  int rc = enter(h);
  if (rc) return rc;
  if (!residual) return fail(PE_EINVAL, "residual is NULL");
  rc = read_stats(h);
  if (rc) return rc;
  std::memcpy(residual, &h->host_stats->residual, sizeof(double));
  return PE_OK;
}

int pe_square_profile(pe_square *h, int32_t enable) {
  int rc = enter(h);
  if (rc) return rc;
  return h->timer.reset(enable != 0);
}

int pe_square_kernel_time(pe_square *h, double *total_ms, int64_t *launches) {
  int rc = enter(h);
  if (rc) return rc;
  if (!total_ms || !launches) return fail(PE_EINVAL, "NULL argument");
  rc = h->timer.harvest(true);
  if (rc) return rc;
  *total_ms = h->timer.ms(0);
  *launches = h->timer.launches(0);
  return PE_OK;
}

int pe_square_destroy(pe_square *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->p.device);
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
