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

// Initial field: TUBE hypot(x, y) - radius; MINTIME 0 inside the capture
// disk and 1 elsewhere.  plane: dense (y, x) values computed on the host.
cudaError_t sl_init(const SLGrid &g, const float *plane, float *field,
                    cudaStream_t stream);

}  // namespace pe
