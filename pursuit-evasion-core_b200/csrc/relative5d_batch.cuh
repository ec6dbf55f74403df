// Batched relative 5D ENO/LF solves: many independent grids of different
// sizes and physics advanced to their own horizons by one persistent
// launch.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "relative5d.cuh"

namespace pe {

// One solve of a batch, in device memory.
struct Rel5BatchSolve {
  Rel5Grid g;
  float *a, *b, *arrival;  // padded fields: value, RK2 stage, arrival time
  const double *sn, *cs;   // heading tables (double)
  const double2 *steps;    // (t, dt) of every RK step, as the reference loop takes them
  Rel5Stats *stats;        // residual of the last step, largest increase, flags
  int nsteps;
  int rows;                // y rows per work item (the tile)
  int64_t items;           // work items of one stage: nvp * nve * nh * ceil(nx / rows)
  int64_t item_base;       // index of the solve's first item in the batch
};

struct Rel5BatchArgs {
  const Rel5BatchSolve *solves;  // sorted by nsteps, longest first
  const int64_t *active_items;   // [max_steps]: items of the solves still
                                 // stepping at step k (a prefix of the batch)
  int count, max_steps;
  unsigned *sync;                // [0] arrivals, [1] generation, [2] timeout flag
};

// Threads per CTA of the batched kernel.
constexpr int kRel5BatchThreads = 256;

// CTAs of one cooperative launch on the current device (all co-resident).
int rel5_batch_grid_exact();

// Every step of every solve (RK2) in one cooperative launch; stages are
// separated by a grid-wide barrier whose waits are bounded (timeout flag
// sync[2]).  `sync` must be zeroed before the launch.  Exact: the
// single-grid exact path's arithmetic (each solve equals it bit for bit).
cudaError_t rel5_batch_run_exact(const Rel5BatchArgs &args, int grid, cudaStream_t stream);

// Float32 update, tiled (relative5d_batch_tiled.cu): a work item is `rows` y
// rows of one (vP, vE) plane stack, all headings, one thread per 4-cell x
// chunk.  rows: the tile clamped to the CTA (want < 1: the largest that
// fits); smem: dynamic shared memory of a CTA for that tile; grid: CTAs of
// one cooperative launch with that shared memory.
int rel5_batch_tiled_rows(int nx, int xp, int want);
size_t rel5_batch_tiled_smem(int rows, int xp);
int rel5_batch_grid_tiled(size_t smem);
cudaError_t rel5_batch_run_tiled(const Rel5BatchArgs &args, int grid, size_t smem,
                                 cudaStream_t stream);

}  // namespace pe
