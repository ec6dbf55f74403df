// C-ABI of the relative 5D semi-Lagrangian solver handle (pe_semilag_*).
//
// The host tabulates, in double, the exact held-command arcs of every
// (speed level, action) pair (reversible/model.py:86-153) and the evader's
// displacement in the pursuer frame for every heading, then drives the
// min-max backups (semilag5d.cu) and the value-iteration loop with a
// sup-norm stopping test.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pe_internal.h"
#include "semilag5d.cuh"

struct pe_semilag {
  pe_semilag_params p{};
  pe::SLGrid g{};
  double dt = 0, dphi = 0, dvp = 0, dve = 0;
  float *a = nullptr, *b = nullptr, *plane = nullptr;
  uint8_t *pol_p = nullptr, *pol_e = nullptr;
  pe::SLPursuerArc *parc = nullptr;
  pe::SLEvaderArc *earc = nullptr;
  pe::SLEvaderMove *emove = nullptr;
  pe::SLStats *stats = nullptr, *host_stats = nullptr;
  // tiled value-only kernel (semilag5d_tiled.cu), when the grid allows it
  pe::SLSpeedStep *pstep = nullptr, *estep = nullptr;
  uint8_t *hint = nullptr;
  pe::SLTiledPlan plan{};
  // per-item change flags of the last two tiled backups (work skipping)
  unsigned *changed[2] = {nullptr, nullptr};
  int changed_cur = 0;       // changed[changed_cur]: the last backup's flags
  bool skip_valid = false;   // ... are those of the field now in `a`
  bool skip_enabled = true;
  int smem_limit = 0;  // dynamic shared memory available to the tiled kernel
  bool tiled_ok = false;    // the tiled kernel applies to this grid and dt
  bool tiled_auto = false;  // ... and has enough work items to be the faster one
  int kernel = PE_SL_KERNEL_AUTO;
  cudaStream_t own = nullptr, stream = nullptr;
  int64_t iterations = 0;
  bool initialized = false, policy_valid = false;
  float *arrival = nullptr;  // first-crossing times (tube mode, when tracked)
  double time = 0;           // start time of the next backup, for the arrival
  pe::LaunchTimer timer;  // launch times (profile / kernel_time)
};

namespace {

using pe::fail;

void speed_arc(double v, double a, double dt, double vmin, double vmax,
               double *v_out, double *dist) {
  // model.py:86-109
  const double target = a >= 0 ? vmax : vmin;
  const double hit = std::fabs(a) > 1e-14 ? (target - v) / a : INFINITY;
  const double active = std::fmin(dt, std::fmax(0.0, hit));
  double final = v + a * dt;
  final = final < vmin ? vmin : (final > vmax ? vmax : final);
  *v_out = final;
  *dist = v * active + 0.5 * a * active * active + final * (dt - active);
}

void chord_turn(double d, double k, double *chord, double *turn) {
  // model.py:144-146: chord = d * sinc(turn / 2pi) = d * sin(turn/2) / (turn/2)
  const double t = k * d, half = 0.5 * t;
  *turn = t;
  *chord = std::fabs(half) < 1e-12 ? d : d * std::sin(half) / half;
}

// Speed interpolation steps of one car (SLSpeedStep) from its arc table
// fv[level * 9 + action]; false if a successor leaves the three slabs
// around its level or the speed depends on the steering.
template <typename Arc>
bool speed_steps(const std::vector<Arc> &arc, int levels, std::vector<pe::SLSpeedStep> *out) {
  out->resize(levels);
  for (int lv = 0; lv < levels; lv++) {
    pe::SLSpeedStep &st = (*out)[lv];
    st.base = std::min(std::max(lv - 1, 0), levels - 3);
    for (int a = 0; a < 3; a++) {
      const float fv = arc[lv * 9 + 3 * a + 1].fv;
      if (arc[lv * 9 + 3 * a].fv != fv || arc[lv * 9 + 3 * a + 2].fv != fv) return false;
      int j = (int)std::floor(fv);
      j = std::min(std::max(j, 0), levels - 2);
      const int slot = j - st.base;
      if (slot < 0 || slot > 1) return false;
      st.slot[a] = slot;
      st.w[a] = fv - (float)j;
    }
  }
  return true;
}

// The tiled kernel stages two halo cells around a tile and one heading
// plane on each side: every successor must stay within 1.99 cells in x and
// y and below one heading spacing.  The displacement is affine in the cell
// position, so its extremes sit at the corners of the position box.
bool tiled_geometry_ok(const pe::SLGrid &g, const std::vector<pe::SLPursuerArc> &parc,
                       const std::vector<pe::SLEvaderArc> &earc,
                       const std::vector<pe::SLEvaderMove> &emove) {
  const double center = 0.5 * (g.nx - 1), ihx = g.ihx;
  double reach = 0, turn = 0;
  for (int iv = 0; iv < g.nvp; iv++)
    for (int up = 0; up < 9; up++) {
      const pe::SLPursuerArc &pa = parc[iv * 9 + up];
      const double rot = (std::fabs(pa.c - 1.0) + std::fabs(pa.s)) * center;
      for (int ie = 0; ie < g.nve; ie++)
        for (int ue = 0; ue < 9; ue++) {
          turn = std::max(turn, std::fabs((double)earc[ie * 9 + ue].turn_idx -
                                          (double)pa.turn_idx));
          for (int ip = 0; ip < g.nh; ip++) {
            const pe::SLEvaderMove &em = emove[((size_t)ip * g.nve + ie) * 9 + ue];
            const double dxp = (double)em.ex - pa.px, dyp = (double)em.ey - pa.py;
            const double ox = std::fabs(pa.c * dxp + pa.s * dyp) * ihx;
            const double oy = std::fabs(pa.c * dyp - pa.s * dxp) * ihx;
            reach = std::max(reach, rot + std::max(ox, oy));
          }
        }
    }
  return reach <= 1.99 && turn < 0.999;
}

int validate(const pe_semilag_params *p) {
  if (!p) return fail(PE_EINVAL, "params is NULL");
  const double v[] = {p->extent, p->capture_radius, p->p_speed_min, p->p_speed_max,
                      p->p_acceleration, p->p_curvature, p->e_speed_min,
                      p->e_speed_max, p->e_acceleration, p->e_curvature, p->dt};
  for (double x : v)
    if (!std::isfinite(x)) return fail(PE_EINVAL, "Invalid solver options: non-finite value");
  if (p->positions < 3 || p->headings < 4 || p->p_speeds < 3 || p->e_speeds < 3 ||
      p->extent <= p->capture_radius || p->capture_radius <= 0 ||
      p->p_acceleration <= 0 || p->e_acceleration <= 0 || p->p_curvature <= 0 ||
      p->e_curvature <= 0 || p->p_speed_min >= p->p_speed_max ||
      p->e_speed_min >= p->e_speed_max || p->dt < 0 ||
      (p->mode != PE_SL_TUBE && p->mode != PE_SL_MINTIME))
    return fail(PE_EINVAL, "Invalid solver options");
  if ((int64_t)p->p_speeds * p->e_speeds > 65535 || p->headings > 65535)
    return fail(PE_EINVAL, "Invalid solver options: grid too large");
  return PE_OK;
}

// Largest dt that moves no coordinate by more than one grid spacing (the
// interpolation CFL), from the same rate bounds as native_relative.cpp:76-81.
double interpolation_cfl_dt(const pe_semilag_params *p) {
  const double pi = std::acos(-1.0);
  const double dx = 2 * p->extent / (p->positions - 1), dphi = 2 * pi / p->headings;
  const double dvp = (p->p_speed_max - p->p_speed_min) / (p->p_speeds - 1);
  const double dve = (p->e_speed_max - p->e_speed_min) / (p->e_speeds - 1);
  const double VP = std::max(std::fabs(p->p_speed_min), std::fabs(p->p_speed_max));
  const double VE = std::max(std::fabs(p->e_speed_min), std::fabs(p->e_speed_max));
  const double rates[5] = {(VP + VE + VP * p->p_curvature * p->extent) / dx,
                           (VE + VP * p->p_curvature * p->extent) / dx,
                           (VP * p->p_curvature + VE * p->e_curvature) / dphi,
                           p->p_acceleration / dvp, p->e_acceleration / dve};
  double worst = 0;
  for (double r : rates) worst = std::max(worst, r);
  return 1.0 / worst;
}

void release(pe_semilag *h) {
  for (void *ptr : {(void *)h->a, (void *)h->b, (void *)h->plane, (void *)h->pol_p,
                    (void *)h->pol_e, (void *)h->parc, (void *)h->earc,
                    (void *)h->emove, (void *)h->stats, (void *)h->pstep,
                    (void *)h->estep, (void *)h->hint, (void *)h->arrival,
                    (void *)h->changed[0], (void *)h->changed[1]})
    cudaFree(ptr);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->own) cudaStreamDestroy(h->own);
}

int enter(pe_semilag *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->p.device));
  return PE_OK;
}

int read_stats(pe_semilag *h) {
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_stats, h->stats, sizeof(pe::SLStats),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->host_stats->nonfinite) return fail(PE_ENONFINITE, "Nonfinite value update");
  return PE_OK;
}

bool use_tiled(const pe_semilag *h) {
  if (h->kernel == PE_SL_KERNEL_TILED) return h->tiled_ok;
  return h->kernel == PE_SL_KERNEL_AUTO && h->tiled_auto;
}

// Reset the per-cell action hints of the tiled kernel (neutral pair).
int reset_hints(pe_semilag *h) {
  if (h->hint) PE_CUDA_TRY(cudaMemsetAsync(h->hint, 0x44, (size_t)h->g.n, h->stream));
  return PE_OK;
}

int backup(pe_semilag *h, bool policy) {
  PE_CUDA_TRY(cudaMemsetAsync(&h->stats->residual, 0, sizeof(unsigned long long),
                              h->stream));
  pe::SLBackup bk{};
  bk.src = h->a;
  bk.dst = h->b;
  bk.policy_p = policy ? h->pol_p : nullptr;
  bk.policy_e = policy ? h->pol_e : nullptr;
  bk.parc = h->parc;
  bk.earc = h->earc;
  bk.emove = h->emove;
  bk.stats = h->stats;
  cudaEvent_t e0 = h->timer.begin(h->stream);
  if (!policy && use_tiled(h)) {
    const bool skip = h->skip_enabled && h->skip_valid;
    const pe::SLTiled tl{h->pstep, h->estep, h->hint,
                         skip ? h->changed[h->changed_cur] : nullptr,
                         h->changed[h->changed_cur ^ 1]};
    PE_CUDA_TRY(pe::sl_backup_tiled(h->g, bk, tl, h->plan, h->stream));
    h->changed_cur ^= 1;
    h->skip_valid = true;
  } else {
    PE_CUDA_TRY(pe::sl_backup(h->g, bk, h->stream));
    h->skip_valid = false;  // the generic kernel keeps no change flags
  }
  pe::count_launches(1);
  {
    const int rc = h->timer.end(h->stream, e0, 0);
    if (rc) return rc;
  }
  std::swap(h->a, h->b);
  if (h->arrival) {
    PE_CUDA_TRY(pe::sl_arrival(h->g, h->b, h->a, h->arrival, h->time, h->dt, h->stream));
    pe::count_launches(1);
  }
  h->time += h->dt;
  h->iterations++;
  h->policy_valid = policy;
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_semilag_dt(const pe_semilag_params *params, double *dt) {
  const int rc = validate(params);
  if (rc) return rc;
  if (!dt) return fail(PE_EINVAL, "dt is NULL");
  *dt = params->dt > 0 ? params->dt : interpolation_cfl_dt(params);
  return PE_OK;
}

int pe_semilag_create(const pe_semilag_params *params, pe_semilag **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  PE_CUDA_TRY(cudaSetDevice(params->device));
  pe_semilag *h = new pe_semilag();
  h->p = *params;
  const double pi = std::acos(-1.0);
  h->dt = params->dt > 0 ? params->dt : interpolation_cfl_dt(params);
  h->dphi = 2 * pi / params->headings;
  h->dvp = (params->p_speed_max - params->p_speed_min) / (params->p_speeds - 1);
  h->dve = (params->e_speed_max - params->e_speed_min) / (params->e_speeds - 1);
  pe::SLGrid &g = h->g;
  g.nx = params->positions;
  g.nh = params->headings;
  g.nvp = params->p_speeds;
  g.nve = params->e_speeds;
  g.mode = params->mode;
  g.sy = g.nx;
  g.sp = (int64_t)g.nx * g.nx;
  g.se = g.sp * g.nh;
  g.sv = g.se * g.nve;
  g.n = g.sv * g.nvp;
  const double dx = 2 * params->extent / (params->positions - 1);
  g.extent = (float)params->extent;
  g.dx = (float)dx;
  g.ihx = (float)(1.0 / dx);
  g.radius = (float)params->capture_radius;
  g.beta = (float)std::exp(-h->dt);
  // Arc tables (double on the host, float on the device).
  std::vector<pe::SLPursuerArc> parc(g.nvp * 9);
  std::vector<pe::SLEvaderArc> earc(g.nve * 9);
  std::vector<pe::SLEvaderMove> emove((size_t)g.nh * g.nve * 9);
  for (int iv = 0; iv < g.nvp; iv++)
    for (int u = 0; u < 9; u++) {
      const double a = (u / 3 - 1) * params->p_acceleration;
      const double k = (u % 3 - 1) * params->p_curvature;
      const double v = params->p_speed_min + iv * h->dvp;
      double v2, d, chord, turn;
      speed_arc(v, a, h->dt, params->p_speed_min, params->p_speed_max, &v2, &d);
      chord_turn(d, k, &chord, &turn);
      pe::SLPursuerArc &e = parc[iv * 9 + u];
      e.px = (float)(chord * std::cos(0.5 * turn));
      e.py = (float)(chord * std::sin(0.5 * turn));
      e.c = (float)std::cos(turn);
      e.s = (float)std::sin(turn);
      e.turn_idx = (float)(turn / h->dphi);
      e.fv = (float)((v2 - params->p_speed_min) / h->dvp);
    }
  for (int ie = 0; ie < g.nve; ie++)
    for (int w = 0; w < 9; w++) {
      const double a = (w / 3 - 1) * params->e_acceleration;
      const double k = (w % 3 - 1) * params->e_curvature;
      const double v = params->e_speed_min + ie * h->dve;
      double v2, d, chord, turn;
      speed_arc(v, a, h->dt, params->e_speed_min, params->e_speed_max, &v2, &d);
      chord_turn(d, k, &chord, &turn);
      earc[ie * 9 + w].turn_idx = (float)(turn / h->dphi);
      earc[ie * 9 + w].fv = (float)((v2 - params->e_speed_min) / h->dve);
      for (int ip = 0; ip < g.nh; ip++) {
        const double psi = -pi + ip * h->dphi;
        pe::SLEvaderMove &m = emove[((size_t)ip * g.nve + ie) * 9 + w];
        m.ex = (float)(chord * std::cos(psi + 0.5 * turn));
        m.ey = (float)(chord * std::sin(psi + 0.5 * turn));
      }
    }
  // tiled value-only kernel: speed steps, geometry and a shared-memory plan
  std::vector<pe::SLSpeedStep> pstep, estep;
  {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                           params->device);
    h->smem_limit = optin - 1024;
    h->tiled_ok = speed_steps(parc, g.nvp, &pstep) && speed_steps(earc, g.nve, &estep) &&
                  tiled_geometry_ok(g, parc, earc, emove) &&
                  pe::sl_tiled_plan(g, optin - 1024, 0, &h->plan);
    // one CTA per SM: with fewer than ~8 items per SM the tail of the last
    // wave and the per-item ring warm-up outweigh the gain (measured on a
    // 33x24x11x11 grid: 1.46 ms tiled vs 0.81 ms generic per backup)
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, params->device);
    h->tiled_auto = h->tiled_ok && h->plan.items >= 8 * (int64_t)sms;
  }
  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  const size_t bytes = sizeof(float) * (size_t)g.n;
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->a, bytes));
  take(cudaMalloc(&h->b, bytes));
  take(cudaMalloc(&h->plane, sizeof(float) * (size_t)g.sp));
  take(cudaMalloc(&h->pol_p, (size_t)g.n));
  take(cudaMalloc(&h->pol_e, (size_t)g.n));
  take(cudaMalloc(&h->parc, sizeof(pe::SLPursuerArc) * parc.size()));
  take(cudaMalloc(&h->earc, sizeof(pe::SLEvaderArc) * earc.size()));
  take(cudaMalloc(&h->emove, sizeof(pe::SLEvaderMove) * emove.size()));
  take(cudaMalloc(&h->stats, sizeof(pe::SLStats)));
  take(cudaMallocHost(&h->host_stats, sizeof(pe::SLStats)));
  if (err == cudaSuccess) {
    take(cudaMemcpy(h->parc, parc.data(), sizeof(pe::SLPursuerArc) * parc.size(),
                    cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->earc, earc.data(), sizeof(pe::SLEvaderArc) * earc.size(),
                    cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->emove, emove.data(), sizeof(pe::SLEvaderMove) * emove.size(),
                    cudaMemcpyHostToDevice));
    take(cudaMemset(h->stats, 0, sizeof(pe::SLStats)));
  }
  if (err == cudaSuccess && h->tiled_ok) {
    take(cudaMalloc(&h->pstep, sizeof(pe::SLSpeedStep) * pstep.size()));
    take(cudaMalloc(&h->estep, sizeof(pe::SLSpeedStep) * estep.size()));
    take(cudaMalloc(&h->hint, (size_t)g.n));
    // flags for the finest possible tiling (one row per tile)
    const size_t flags = sizeof(unsigned) * (size_t)g.nvp * g.nve * g.nx;
    take(cudaMalloc(&h->changed[0], flags));
    take(cudaMalloc(&h->changed[1], flags));
    if (err == cudaSuccess) {
      take(cudaMemcpy(h->pstep, pstep.data(), sizeof(pe::SLSpeedStep) * pstep.size(),
                      cudaMemcpyHostToDevice));
      take(cudaMemcpy(h->estep, estep.data(), sizeof(pe::SLSpeedStep) * estep.size(),
                      cudaMemcpyHostToDevice));
    }
  }
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_semilag_create");
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_semilag_init(pe_semilag *h, const float *initial) {
  int rc = enter(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::SLStats), h->stream));
  if (initial) {
    PE_CUDA_TRY(cudaMemcpyAsync(h->a, initial, sizeof(float) * (size_t)h->g.n,
                                cudaMemcpyHostToDevice, h->stream));
  } else {
    const int nx = h->g.nx;
    const double dx = 2 * h->p.extent / (nx - 1);
    std::vector<float> plane((size_t)nx * nx);
    for (int iy = 0; iy < nx; iy++)
      for (int ix = 0; ix < nx; ix++) {
        const double d = std::hypot(-h->p.extent + ix * dx, -h->p.extent + iy * dx) -
                         h->p.capture_radius;
        plane[(size_t)iy * nx + ix] =
            h->p.mode == PE_SL_TUBE ? (float)d : (d <= 0 ? 0.f : 1.f);
      }
    PE_CUDA_TRY(cudaMemcpyAsync(h->plane, plane.data(), sizeof(float) * plane.size(),
                                cudaMemcpyHostToDevice, h->stream));
    PE_CUDA_TRY(pe::sl_init(h->g, h->plane, h->a, h->stream));
    pe::count_launches(1);
  }
  rc = reset_hints(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->iterations = 0;
  h->initialized = true;
  h->policy_valid = false;
  h->skip_valid = false;
  return PE_OK;
}

int pe_semilag_init_device(pe_semilag *h, const float *device_initial) {
  int rc = enter(h);
  if (rc) return rc;
  if (!device_initial) return fail(PE_EINVAL, "device_initial is NULL");
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::SLStats), h->stream));
  PE_CUDA_TRY(cudaMemcpyAsync(h->a, device_initial, sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToDevice, h->stream));
  rc = reset_hints(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->iterations = 0;
  h->initialized = true;
  h->policy_valid = false;
  h->skip_valid = false;
  return PE_OK;
}

int pe_semilag_backup(pe_semilag *h, int with_policy) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "backup before init");
  return backup(h, with_policy != 0);
}

int pe_semilag_iterate(pe_semilag *h, int64_t max_iterations, double tol,
                       int32_t check_every, int64_t *iterations,
                       double *residual, int32_t *converged) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "iterate before init");
  if (max_iterations < 0 || !(tol >= 0) || check_every < 1)
    return fail(PE_EINVAL, "max_iterations >= 0, tol >= 0, check_every >= 1");
  int64_t done = 0;
  double r = INFINITY;
  int conv = 0;
  while (done < max_iterations) {
    rc = backup(h, false);
    if (rc) return rc;
    done++;
    if (done % check_every == 0 || done == max_iterations) {
      rc = read_stats(h);
      if (rc) return rc;
      std::memcpy(&r, &h->host_stats->residual, sizeof r);
      if (tol > 0 && r < tol) {
        conv = 1;
        break;
      }
    }
  }
  if (iterations) *iterations = done;
  if (residual) *residual = r;
  if (converged) *converged = conv;
  return PE_OK;
}

int pe_semilag_residual(pe_semilag *h, double *residual) {
  int rc = enter(h);
  if (rc) return rc;
  rc = read_stats(h);
  if (rc) return rc;
  if (residual) std::memcpy(residual, &h->host_stats->residual, sizeof(double));
  return PE_OK;
}

int pe_semilag_evaluations(pe_semilag *h, int64_t *evaluations) {
  int rc = enter(h);
  if (rc) return rc;
  if (!evaluations) return fail(PE_EINVAL, "evaluations is NULL");
  rc = read_stats(h);
  if (rc) return rc;
  *evaluations = (int64_t)h->host_stats->evaluations;
  return PE_OK;
}

int pe_semilag_set_skip(pe_semilag *h, int enable) {
  int rc = enter(h);
  if (rc) return rc;
  h->skip_enabled = enable != 0;
  return PE_OK;
}

int pe_semilag_items_computed(pe_semilag *h, int64_t *items) {
  int rc = enter(h);
  if (rc) return rc;
  if (!items) return fail(PE_EINVAL, "items is NULL");
  rc = read_stats(h);
  if (rc) return rc;
  *items = (int64_t)h->host_stats->items_computed;
  return PE_OK;
}

int pe_semilag_copy_value(pe_semilag *h, float *host_value) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_value) return fail(PE_EINVAL, "host_value is NULL");
  PE_CUDA_TRY(cudaMemcpyAsync(host_value, h->a, sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_semilag_copy_value_device(pe_semilag *h, float *device_value) {
  int rc = enter(h);
  if (rc) return rc;
  if (!device_value) return fail(PE_EINVAL, "device_value is NULL");
  PE_CUDA_TRY(cudaMemcpyAsync(device_value, h->a, sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToDevice, h->stream));
  return read_stats(h);
}

int pe_semilag_copy_policy(pe_semilag *h, uint8_t *host_p, uint8_t *host_e) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->policy_valid)
    return fail(PE_ESTATE, "no policy: run pe_semilag_backup(h, 1) first");
  if (host_p)
    PE_CUDA_TRY(cudaMemcpyAsync(host_p, h->pol_p, (size_t)h->g.n,
                                cudaMemcpyDeviceToHost, h->stream));
  if (host_e)
    PE_CUDA_TRY(cudaMemcpyAsync(host_e, h->pol_e, (size_t)h->g.n,
                                cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

int pe_semilag_device_value(pe_semilag *h, float **device_value) {
  if (!h || !device_value) return fail(PE_EINVAL, "NULL argument");
  *device_value = h->a;
  return PE_OK;
}

int pe_semilag_iterations(const pe_semilag *h, int64_t *iterations) {
  if (!h || !iterations) return fail(PE_EINVAL, "NULL argument");
  *iterations = h->iterations;
  return PE_OK;
}

int pe_semilag_set_stream(pe_semilag *h, void *cuda_stream) {
  int rc = enter(h);
  if (rc) return rc;
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own;
  return PE_OK;
}

int pe_semilag_set_kernel(pe_semilag *h, int kernel) {
  int rc = enter(h);
  if (rc) return rc;
  if (kernel != PE_SL_KERNEL_AUTO && kernel != PE_SL_KERNEL_GENERIC &&
      kernel != PE_SL_KERNEL_TILED)
    return fail(PE_EINVAL, "unknown backup kernel %d", kernel);
  if (kernel == PE_SL_KERNEL_TILED && !h->tiled_ok)
    return fail(PE_EINVAL, "the tiled backup kernel does not apply to this grid and dt");
  h->kernel = kernel;
  return PE_OK;
}

int pe_semilag_set_tile(pe_semilag *h, int32_t rows) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->tiled_ok) return fail(PE_EINVAL, "the tiled backup kernel does not apply");
  pe::SLTiledPlan plan{};
  if (rows < 0 || !pe::sl_tiled_plan(h->g, h->smem_limit, rows, &plan))
    return fail(PE_EINVAL, "tile of %d rows does not fit the tiled kernel", rows);
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->plan = plan;
  h->skip_valid = false;  // the flags index the old tiling
  return PE_OK;
}

int pe_semilag_get_tile(const pe_semilag *h, int32_t *rows, int32_t *threads,
                        int64_t *items) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (rows) *rows = h->tiled_ok ? h->plan.rows : 0;
  if (threads) *threads = h->tiled_ok ? h->plan.threads : 0;
  if (items) *items = h->tiled_ok ? h->plan.items : 0;
  return PE_OK;
}

int pe_semilag_kernel(const pe_semilag *h, int32_t *kernel) {
  if (!h || !kernel) return fail(PE_EINVAL, "handle or kernel is NULL");
  *kernel = use_tiled(h) ? PE_SL_KERNEL_TILED : PE_SL_KERNEL_GENERIC;
  return PE_OK;
}

int pe_semilag_profile(pe_semilag *h, int enable) {
  int rc = enter(h);
  if (rc) return rc;
  return h->timer.reset(enable != 0);
}

int pe_semilag_kernel_time(pe_semilag *h, double *total_ms, int64_t *launches) {
  int rc = enter(h);
  if (rc) return rc;
  rc = h->timer.harvest(true);
  if (rc) return rc;
  if (total_ms) *total_ms = h->timer.ms(0);
  if (launches) *launches = h->timer.launches(0);
  return PE_OK;
}

int pe_semilag_track_arrival(pe_semilag *h, const float *host_arrival, double start_time) {
  int rc = enter(h);
  if (rc) return rc;
  if (h->p.mode != PE_SL_TUBE) return fail(PE_EINVAL, "arrival times need the tube mode");
  if (!h->initialized) return fail(PE_ESTATE, "track_arrival before init");
  if (!std::isfinite(start_time)) return fail(PE_EINVAL, "start_time must be finite");
  const size_t bytes = sizeof(float) * (size_t)h->g.n;
  if (!h->arrival) PE_CUDA_TRY(cudaMalloc(&h->arrival, bytes));
  if (host_arrival) {
    PE_CUDA_TRY(cudaMemcpyAsync(h->arrival, host_arrival, bytes, cudaMemcpyHostToDevice,
                                h->stream));
  } else {
    // arrival = start_time where the value is <= 0, NaN elsewhere
    PE_CUDA_TRY(pe::sl_arrival_start(h->g, h->a, h->arrival, start_time, h->stream));
    pe::count_launches(1);
  }
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->time = start_time;
  return PE_OK;
}

int pe_semilag_copy_arrival(pe_semilag *h, float *host_arrival) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_arrival) return fail(PE_EINVAL, "host_arrival is NULL");
  if (!h->arrival) return fail(PE_ESTATE, "arrival is not tracked");
  PE_CUDA_TRY(cudaMemcpyAsync(host_arrival, h->arrival, sizeof(float) * (size_t)h->g.n,
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_semilag_destroy(pe_semilag *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
