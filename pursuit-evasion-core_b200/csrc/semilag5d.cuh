// Relative 5D semi-Lagrangian min-max backup: shared declarations.
//
// Dense storage [vP, vE, psi, y, x], x fastest.  One backup = for every
// cell, the minimum over the 9 pursuer actions of the maximum over the 9
// evader actions of the value interpolated (5D multilinear) at the exact
// held-command successor after dt.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pe {

enum { SL_TUBE = 0, SL_MINTIME = 1 };

struct SLGrid {
  int nx, nh, nvp, nve, mode;
  int64_t n, sy, sp, se, sv;
  float extent, dx, ihx, radius, beta;  // beta = exp(-dt) (MINTIME)
};

// Per (speed level, action) arc tables, computed on the host in double.
struct SLPursuerArc {  // [nvp][9]
  float px, py, c, s;  // pursuer displacement, cos/sin of its turn
  float turn_idx;      // turn / dphi
  float fv;            // (v' - v_lo) / dv, exact grid index of the new speed
};
struct SLEvaderArc {  // [nve][9]
  float turn_idx;     // turn / dphi
  float fv;           // (v' - v_lo) / dv
};
struct SLEvaderMove {  // [nh][nve][9]: evader displacement in the P frame
  float ex, ey;
};

struct SLStats {
  unsigned long long residual;  // bits of a non-negative double
  unsigned int nonfinite;
  unsigned int pad;
  // interpolated action-pair evaluations of the tiled kernel's live cells
  // (probes, full reply scans and pruned replies) since the last reset
  unsigned long long evaluations;
  // work items of the tiled kernel computed (not skipped) since the last reset
  unsigned long long items_computed;
};

struct SLBackup {
  const float *src;
  float *dst;
  uint8_t *policy_p, *policy_e;  // nullptr: value only (pursuer pruning on)
  const SLPursuerArc *parc;
  const SLEvaderArc *earc;
  const SLEvaderMove *emove;
  SLStats *stats;
};

cudaError_t sl_backup(const SLGrid &g, const SLBackup &b, cudaStream_t stream);

// ---- shared-memory tiled backup (semilag5d_tiled.cu), value only ----------

#define SL_TILED_MAX_THREADS 512

// Speed interpolation of one car's successors from one speed level: the
// three staged slabs are base, base+1, base+2; acceleration index a blends
// slab base+slot[a] and the next one with upper weight w[a].
struct SLSpeedStep {
  int base;
  int slot[3];
  float w[3];
};

struct SLTiled {
  const SLSpeedStep *pstep;  // [nvp]
  const SLSpeedStep *estep;  // [nve]
  uint8_t *hint;             // [cells]: (pursuer action << 4) | evader reply of
                             // the previous backup; 0x44 before the first
  // Work skipping: changed_in[item] != 0 where some cell of the item changed
  // (in its bits) in the previous backup; an item whose 3x3x3 neighbourhood
  // of items (vP, vE, y tile +-1) did not change reads the same inputs as
  // then, so its cells are copied instead of recomputed.  nullptr: every
  // item is computed.  changed_out (may be nullptr) receives this backup's
  // flags.
  const unsigned *changed_in;
  unsigned *changed_out;
};

struct SLTiledPlan {
  int rows;        // cell rows of a tile (full x width)
  int tiles_y;
  int psi_chunk, psi_chunks;
  int threads;
  int64_t items;   // nvp * nve * tiles_y * psi_chunks
  size_t smem;     // dynamic shared memory per CTA
};

// Tile plan for grid g within max_smem bytes of dynamic shared memory
// (want_rows > 0: about that many cell rows per tile, else the default);
// false if the grid's width or the tile does not fit the tiled kernel.
bool sl_tiled_plan(const SLGrid &g, int max_smem, int want_rows, SLTiledPlan *plan);

cudaError_t sl_backup_tiled(const SLGrid &g, const SLBackup &b, const SLTiled &t,
                            const SLTiledPlan &plan, cudaStream_t stream);

// Initial field: TUBE hypot(x, y) - radius; MINTIME 0 inside the capture
// disk and 1 elsewhere.  plane: dense (y, x) values computed on the host.
// First crossing of zero between two tube values (the arrival rule of the
// ENO/LF path, native_relative.cpp:167-168): where prev > 0 >= cur and the
// arrival is still NaN, arrival = t + dt * prev / (prev - cur).
cudaError_t sl_arrival(const SLGrid &g, const float *prev, const float *cur, float *arrival,
                       double t, double dt, cudaStream_t stream);
// arrival = start_time where cur <= 0, NaN elsewhere.
cudaError_t sl_arrival_start(const SLGrid &g, const float *cur, float *arrival,
                             double start_time, cudaStream_t stream);

cudaError_t sl_init(const SLGrid &g, const float *plane, float *field,
                    cudaStream_t stream);

}  // namespace pe
