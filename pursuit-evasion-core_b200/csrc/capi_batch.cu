// C-ABI of the batched relative 5D solver (pe_batch_*): many independent
// RelativeGrid solves, each with its own grid, physics and horizon, advanced
// together by one persistent cooperative kernel (relative5d_batch_*.cu)
// captured once in a CUDA graph.
//
// Every solve follows the reference executable's driver
// (native_relative.cpp:173-190: steps of min(cfl_limit, horizon - t) until
// t reaches the horizon).  With PE_LOCAL_F64 each solve's field and arrival
// times equal those of a single-grid PE_LOCAL_F64 handle, and the reference
// executable's, bit for bit; PE_LOCAL_F32 runs the float32 cell update.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "pe_internal.h"
#include "relative5d.cuh"
#include "relative5d_batch.cuh"
#include "relative5d_host.h"

struct pe_batch {
  int count = 0;
  int device = 0;
  bool exact = true;
  std::vector<pe_relative_params> params;  // caller's order
  std::vector<double> horizons;
  std::vector<pe::Rel5Grid> grids;
  std::vector<double> limits;
  std::vector<std::vector<double2>> steps;
  std::vector<int> rows;   // tile of every solve (caller's order)
  std::vector<int> order;  // batch position -> caller index (longest first)
  int max_steps = 0;
  // device memory
  float *fields = nullptr;  // per solve: a, b, arrival (padded)
  std::vector<size_t> field_off;
  double *tables = nullptr;  // per solve: sn, cs
  std::vector<size_t> table_off;
  double2 *step_table = nullptr;
  std::vector<size_t> step_off;
  pe::Rel5Stats *stats = nullptr, *host_stats = nullptr;
  pe::Rel5BatchSolve *solves = nullptr;
  int64_t *active_items = nullptr;
  unsigned *sync = nullptr, *host_sync = nullptr;
  float *planes = nullptr;  // capture planes for init
  std::vector<size_t> plane_off;
  cudaStream_t own = nullptr, stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  int grid = 0;
  size_t tiled_smem = 0;  // dynamic shared memory of the tiled float32 kernel
  bool initialized = false;
  pe::LaunchTimer timer;
};

namespace {

using pe::fail;

float *field_a(pe_batch *h, int i) { return h->fields + h->field_off[i]; }
float *field_b(pe_batch *h, int i) { return field_a(h, i) + h->grids[i].n_padded; }
float *field_arrival(pe_batch *h, int i) { return field_b(h, i) + h->grids[i].n_padded; }

void release(pe_batch *h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (void *p : {(void *)h->fields, (void *)h->tables, (void *)h->step_table,
                  (void *)h->stats, (void *)h->solves, (void *)h->active_items,
                  (void *)h->sync, (void *)h->planes})
    cudaFree(p);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->host_sync) cudaFreeHost(h->host_sync);
  if (h->own) cudaStreamDestroy(h->own);
}

int enter(pe_batch *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  return PE_OK;
}

int check_solve(const pe_batch *h, int32_t solve) {
  if (solve < 0 || solve >= h->count)
    return fail(PE_EINVAL, "solve %d out of range (batch of %d)", solve, h->count);
  return PE_OK;
}

// Descriptors and the active-item prefix for the current tiles.
int upload_descriptors(pe_batch *h) {
  std::vector<pe::Rel5BatchSolve> d(h->count);
  int64_t base = 0;
  size_t smem = 0;
  for (int pos = 0; pos < h->count; pos++) {
    const int i = h->order[pos];
    const pe::Rel5Grid &g = h->grids[i];
    pe::Rel5BatchSolve &s = d[pos];
    s.g = g;
    s.a = field_a(h, i);
    s.b = field_b(h, i);
    s.arrival = field_arrival(h, i);
    s.sn = h->tables + h->table_off[i];
    s.cs = s.sn + g.nh;
    s.steps = h->step_table + h->step_off[i];
    s.stats = h->stats + i;
    s.nsteps = (int)h->steps[i].size();
    if (h->exact) {
      // item: `rows` y rows of one (vP, vE, psi) plane
      s.rows = h->rows[i];
      s.items = (int64_t)g.nvp * g.nve * g.nh * ((g.nx + s.rows - 1) / s.rows);
    } else {
      // item: `rows` y rows of one (vP, vE) plane stack, all headings
      s.rows = pe::rel5_batch_tiled_rows(g.nx, g.xp, h->rows[i]);
      s.items = (int64_t)g.nvp * g.nve * ((g.nx + s.rows - 1) / s.rows);
      smem = std::max(smem, pe::rel5_batch_tiled_smem(s.rows, g.xp));
    }
    s.item_base = base;
    base += s.items;
  }
  if (!h->exact && smem != h->tiled_smem) {
    // a different launch shape: size the cooperative grid again and record
    // a new graph at the next run
    h->tiled_smem = smem;
    h->grid = pe::rel5_batch_grid_tiled(smem);
    if (h->grid <= 0) return fail(PE_EINVAL, "batch tiles do not fit the tiled kernel");
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  }
  std::vector<int64_t> active(std::max(h->max_steps, 1), 0);
  for (int k = 0; k < h->max_steps; k++) {
    int64_t n = 0;
    for (int pos = 0; pos < h->count && d[pos].nsteps > k; pos++) n += d[pos].items;
    active[k] = n;
  }
  PE_CUDA_TRY(cudaMemcpyAsync(h->solves, d.data(), sizeof(pe::Rel5BatchSolve) * d.size(),
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaMemcpyAsync(h->active_items, active.data(), sizeof(int64_t) * active.size(),
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

// Record the run (clear the barrier words, then the persistent kernel) as
// a CUDA graph on the handle's stream.
int capture(pe_batch *h) {
  if (h->graph && h->graph_stream == h->stream) return PE_OK;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  pe::Rel5BatchArgs args{};
  args.solves = h->solves;
  args.active_items = h->active_items;
  args.count = h->count;
  args.max_steps = h->max_steps;
  args.sync = h->sync;
  cudaGraph_t g = nullptr;
  PE_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaMemsetAsync(h->sync, 0, 4 * sizeof(unsigned), h->stream);
  if (err == cudaSuccess)
    err = h->exact ? pe::rel5_batch_run_exact(args, h->grid, h->stream)
                   : pe::rel5_batch_run_tiled(args, h->grid, h->tiled_smem, h->stream);
  cudaError_t end = cudaStreamEndCapture(h->stream, &g);
  if (err == cudaSuccess) err = end;
  if (err == cudaSuccess) err = cudaGraphInstantiate(&h->graph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (err != cudaSuccess) return pe::cuda_fail(err, "batch graph capture");
  h->graph_stream = h->stream;
  return PE_OK;
}

int copy_out(pe_batch *h, int32_t solve, float *host, bool arrival) {
  int rc = enter(h);
  if (rc) return rc;
  rc = check_solve(h, solve);
  if (rc) return rc;
  if (!host) return fail(PE_EINVAL, "host buffer is NULL");
  const pe::Rel5Grid &g = h->grids[solve];
  // the stage buffer b is free once a run is complete: pack into it
  float *dense = field_b(h, solve);
  PE_CUDA_TRY(pe::rel5_pack(g, arrival ? field_arrival(h, solve) : field_a(h, solve), dense,
                            h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaMemcpyAsync(host, dense, sizeof(float) * (size_t)g.n,
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_batch_create(const pe_relative_params *params, const double *horizons, int32_t count,
                    int32_t device, pe_batch **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  if (!params || !horizons || count <= 0) return fail(PE_EINVAL, "empty batch");
  for (int i = 0; i < count; i++) {
    const int rc = pe::rel5host::validate(&params[i]);
    if (rc) return fail(rc, "solve %d: %s", i, pe::last_error().c_str());
    if (params[i].order != 2)
      return fail(PE_EINVAL, "solve %d: batched solves are RK2 (order 2)", i);
    if (params[i].precision != params[0].precision)
      return fail(PE_EINVAL, "solve %d: every solve of a batch has the same precision", i);
    if (!(horizons[i] > 0) || !std::isfinite(horizons[i]))
      return fail(PE_EINVAL, "solve %d: horizon must be finite and > 0", i);
  }
  PE_CUDA_TRY(cudaSetDevice(device));
  pe_batch *h = new pe_batch();
  h->count = count;
  h->device = device;
  h->exact = params[0].precision == PE_LOCAL_F64;
  h->params.assign(params, params + count);
  h->horizons.assign(horizons, horizons + count);
  size_t fields = 0, tables = 0, steps = 0, planes = 0;
  for (int i = 0; i < count; i++) {
    const pe::Rel5Grid g = pe::rel5host::make_grid(&params[i]);
    h->grids.push_back(g);
    const double limit = pe::rel5host::cfl_limit(&params[i], g);
    h->limits.push_back(limit);
    std::vector<double2> st;
    double t = 0;
    while (t < horizons[i] - 1e-12) {
      const double dt = std::min(limit, horizons[i] - t);
      st.push_back(make_double2(t, dt));
      t += dt;
    }
    h->max_steps = std::max(h->max_steps, (int)st.size());
    h->steps.push_back(std::move(st));
    // default tile: about one cell per thread (exact), the widest item the
    // CTA holds (tiled float32)
    h->rows.push_back(h->exact ? std::max(1, std::min(g.nx, (256 + g.nx - 1) / g.nx))
                               : pe::rel5_batch_tiled_rows(g.nx, g.xp, 0));
    h->field_off.push_back(fields);
    fields += 3 * (size_t)g.n_padded;
    h->table_off.push_back(tables);
    tables += 2 * (size_t)g.nh;
    h->step_off.push_back(steps);
    steps += h->steps.back().size();
    h->plane_off.push_back(planes);
    planes += (size_t)g.nx * g.nx;
  }
  h->order.resize(count);
  std::iota(h->order.begin(), h->order.end(), 0);
  std::stable_sort(h->order.begin(), h->order.end(), [&](int x, int y) {
    return h->steps[x].size() > h->steps[y].size();
  });

  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->fields, sizeof(float) * fields));
  take(cudaMalloc(&h->tables, sizeof(double) * tables));
  take(cudaMalloc(&h->step_table, sizeof(double2) * std::max<size_t>(steps, 1)));
  take(cudaMalloc(&h->stats, sizeof(pe::Rel5Stats) * count));
  take(cudaMallocHost(&h->host_stats, sizeof(pe::Rel5Stats) * count));
  take(cudaMalloc(&h->solves, sizeof(pe::Rel5BatchSolve) * count));
  take(cudaMalloc(&h->active_items, sizeof(int64_t) * std::max(h->max_steps, 1)));
  take(cudaMalloc(&h->sync, 4 * sizeof(unsigned)));
  take(cudaMallocHost(&h->host_sync, 4 * sizeof(unsigned)));
  take(cudaMalloc(&h->planes, sizeof(float) * planes));
  if (err == cudaSuccess) {
    std::vector<double> tab(tables);
    std::vector<double2> stab(std::max<size_t>(steps, 1));
    std::vector<float> pl(planes);
    for (int i = 0; i < count; i++) {
      std::vector<double> sn, cs;
      pe::rel5host::heading_tables(h->grids[i], &sn, &cs);
      std::copy(sn.begin(), sn.end(), tab.begin() + h->table_off[i]);
      std::copy(cs.begin(), cs.end(), tab.begin() + h->table_off[i] + h->grids[i].nh);
      std::copy(h->steps[i].begin(), h->steps[i].end(), stab.begin() + h->step_off[i]);
      pe::rel5host::capture_plane(h->grids[i], params[i].capture_radius,
                                  pl.data() + h->plane_off[i]);
    }
    take(cudaMemcpy(h->tables, tab.data(), sizeof(double) * tables, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->step_table, stab.data(), sizeof(double2) * stab.size(),
                    cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->planes, pl.data(), sizeof(float) * planes, cudaMemcpyHostToDevice));
    take(cudaMemset(h->stats, 0, sizeof(pe::Rel5Stats) * count));
    take(cudaMemset(h->sync, 0, 4 * sizeof(unsigned)));
  }
  if (err == cudaSuccess) {
    if (h->exact) {  // the tiled kernel's grid is sized with its tiles
      h->grid = pe::rel5_batch_grid_exact();
      if (h->grid <= 0) err = cudaErrorInvalidConfiguration;
    }
  }
  int rc = PE_OK;
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_batch_create");
  } else {
    rc = upload_descriptors(h);
  }
  if (rc) {
    release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_batch_set_tile(pe_batch *h, int32_t solve, int32_t rows) {
  int rc = enter(h);
  if (rc) return rc;
  rc = check_solve(h, solve);
  if (rc) return rc;
  if (rows < 1 || rows > h->grids[solve].nx)
    return fail(PE_EINVAL, "rows must be in [1, positions]");
  h->rows[solve] = rows;
  return upload_descriptors(h);
}

int pe_batch_get_tile(const pe_batch *h, int32_t solve, int32_t *rows) {
  if (!h || !rows) return fail(PE_EINVAL, "handle or rows is NULL");
  const int rc = check_solve(h, solve);
  if (rc) return rc;
  *rows = h->rows[solve];
  return PE_OK;
}

int pe_batch_set_stream(pe_batch *h, void *cuda_stream) {
  int rc = enter(h);
  if (rc) return rc;
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own;
  return PE_OK;
}

int pe_batch_init(pe_batch *h) {
  int rc = enter(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::Rel5Stats) * h->count, h->stream));
  for (int i = 0; i < h->count; i++) {
    PE_CUDA_TRY(pe::rel5_init(h->grids[i], h->planes + h->plane_off[i], field_a(h, i),
                              field_arrival(h, i), 0.f, h->stream));
    pe::count_launches(1);
  }
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->initialized = true;
  return PE_OK;
}

int pe_batch_run(pe_batch *h) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "run before init");
  rc = capture(h);
  if (rc) return rc;
  cudaEvent_t e0 = h->timer.begin(h->stream);
  PE_CUDA_TRY(cudaGraphLaunch(h->graph, h->stream));
  pe::count_launches(1);
  h->initialized = false;  // the fields now hold the solutions
  return h->timer.end(h->stream, e0, 0);
}

int pe_batch_synchronize(pe_batch *h) {
  int rc = enter(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_sync, h->sync, 4 * sizeof(unsigned),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_stats, h->stats, sizeof(pe::Rel5Stats) * h->count,
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->host_sync[2]) return fail(PE_ETIMEOUT, "batch: a bounded device wait (grid barrier or staged heading) gave up");
  for (int i = 0; i < h->count; i++)
    if (h->host_stats[i].nonfinite)
      return fail(PE_ENONFINITE, "batch: non-finite field update in solve %d", i);
  return PE_OK;
}

int pe_batch_solve_info(const pe_batch *h, int32_t solve, int64_t *cells, int64_t *steps,
                        double *dt_limit) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  const int rc = check_solve(h, solve);
  if (rc) return rc;
  if (cells) *cells = h->grids[solve].n;
  if (steps) *steps = (int64_t)h->steps[solve].size();
  if (dt_limit) *dt_limit = h->limits[solve];
  return PE_OK;
}

int pe_batch_copy_field(pe_batch *h, int32_t solve, float *host_field) {
  return copy_out(h, solve, host_field, false);
}

int pe_batch_copy_arrival(pe_batch *h, int32_t solve, float *host_arrival) {
  return copy_out(h, solve, host_arrival, true);
}

int pe_batch_stats(pe_batch *h, int32_t solve, double *residual, double *max_increase) {
  int rc = pe_batch_synchronize(h);
  if (rc) return rc;
  rc = check_solve(h, solve);
  if (rc) return rc;
  double r, inc;
  std::memcpy(&r, &h->host_stats[solve].residual, sizeof r);
  std::memcpy(&inc, &h->host_stats[solve].increase, sizeof inc);
  if (residual) *residual = r;
  if (max_increase) *max_increase = inc;
  return PE_OK;
}

int pe_batch_launch_info(const pe_batch *h, int32_t *ctas, int32_t *threads,
                         int32_t *max_steps, int64_t *total_cell_stages) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  if (ctas) *ctas = h->grid;
  if (threads) *threads = pe::kRel5BatchThreads;
  if (max_steps) *max_steps = h->max_steps;
  if (total_cell_stages) {
    int64_t t = 0;
    for (int i = 0; i < h->count; i++) t += 2 * h->grids[i].n * (int64_t)h->steps[i].size();
    *total_cell_stages = t;
  }
  return PE_OK;
}

int pe_batch_profile(pe_batch *h, int enable) {
  int rc = enter(h);
  if (rc) return rc;
  return h->timer.reset(enable != 0);
}

int pe_batch_kernel_time(pe_batch *h, double *total_ms, int64_t *launches) {
  int rc = enter(h);
  if (rc) return rc;
  rc = h->timer.harvest(true);
  if (rc) return rc;
  if (total_ms) *total_ms = h->timer.ms(0);
  if (launches) *launches = h->timer.launches(0);
  return PE_OK;
}

int pe_batch_destroy(pe_batch *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
