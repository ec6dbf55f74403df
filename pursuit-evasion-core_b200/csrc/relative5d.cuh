// Relative 5D ENO/Lax-Friedrichs capture-tube kernels: shared declarations.
//
// Device layout: the reference's storage order [vP, vE, psi, y, x]
// (free_dp.py:45-54) with every x row padded to `xp` floats (a multiple of 4)
// so that rows, planes and 4-cell chunks are 16-byte aligned for bulk async
// copies and vector loads.  Pad lanes hold 0.  Host copies convert between
// this pitched layout and the dense table layout.
//
// One stage launch = one stage of the RK1/RK2 update of
// native_relative.cpp:124-172 over every cell.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pe {

struct Rel5Grid {
  int nx, nh, nvp, nve, order;
  int xp;                  // padded row length (floats), multiple of 4
  int64_t n;               // cells (dense)
  int64_t n_padded;        // floats of one padded field
  int64_t sy, sp, se, sv;  // padded strides of y, psi, vE, vP (x stride 1)
  double extent, dx, dphi, dvp, dve;
  double vp_lo, ve_lo, acc_p, acc_e, curv_p, curv_e;
  // vP-slab shard: the stage updates global slabs
  // [own_lo, own_lo + own_n) of a buffer whose first slab is global slab
  // slab_lo; own_n == 0 means the whole grid in one buffer
  int own_lo, own_n, slab_lo;
  // 1/h and 1/(h*h) of each axis, rounded to nearest (set_reciprocals):
  // the exact stage's divisions by the spacings go through them
  double rdx, rdx2, rdphi, rdphi2, rdvp, rdvp2, rdve, rdve2;
};

// The reciprocals of a grid's spacings and of their squares (the squares
// rounded as the exact stage forms them, h * h).
inline void set_reciprocals(Rel5Grid &g) {
  g.rdx = 1.0 / g.dx;
  g.rdx2 = 1.0 / (g.dx * g.dx);
  g.rdphi = 1.0 / g.dphi;
  g.rdphi2 = 1.0 / (g.dphi * g.dphi);
  g.rdvp = 1.0 / g.dvp;
  g.rdvp2 = 1.0 / (g.dvp * g.dvp);
  g.rdve = 1.0 / g.dve;
  g.rdve2 = 1.0 / (g.dve * g.dve);
}

// Device-side reduction words of one handle.
struct Rel5Stats {
  unsigned long long residual;  // bits of a non-negative double
  unsigned long long increase;  // bits of a non-negative double
  unsigned int nonfinite;       // set when an update is not finite
  unsigned int timeout;         // set when a bounded device wait gave up
};

struct Rel5Stage {
  const float *src;  // stage input
  float *dst;        // stage output (stage 2: also holds the step's old V)
  // the same for the double-storage stage (rel5_stage_f64_storage)
  const double *src64;
  double *dst64;
  float *arrival;    // first-crossing time, NaN until the cell enters (padded)
  const double *sn, *cs;   // sin/cos of the heading axis, double
  const float *snf, *csf;  // the same, rounded to float
  double dt, t;            // step size and the step's start time
  Rel5Stats *stats;
  // local exit (gpu_relative.py:96-101): cells with x^2 + y^2 > exit_r2 are
  // set to exit_r and never arrive; exit_r2 = 0 disables it
  double exit_r, exit_r2;
  // the same exit as kept x ranges per y row, [lo, hi] (float32 kernels;
  // nullptr when there is no exit)
  const int2 *exit_keep;
};

// Tiling of the fast stage kernel: a CTA owns `rows` y-rows of one (vP, vE)
// plane stack and sweeps `psi_chunk` consecutive headings.
struct Rel5Tile {
  int rows;       // y rows per CTA
  int psi_chunk;  // headings per CTA
};

// Shared memory the fast kernel needs for a tile.
size_t rel5_fast_smem_bytes(const Rel5Grid &g, const Rel5Tile &t);

// Default tile for a grid (rows chosen so rows * xp/4 threads ~ 256).
Rel5Tile rel5_default_tile(const Rel5Grid &g);

// Resident CTAs per SM of the most recent fast-stage launch.
int rel5_last_resident_ctas();

// Whether a tile fits the kernel's limits (threads, shared memory).
bool rel5_tile_valid(const Rel5Grid &g, const Rel5Tile &t);

// Fast path: float32 local arithmetic.  blend = 0 for stage 1 (or the only
// stage of RK1), 1 for the RK2 averaging stage.
cudaError_t rel5_stage_f32(const Rel5Grid &g, const Rel5Tile &t,
                           const Rel5Stage &s, int blend, cudaStream_t stream);

// Exact path: double local arithmetic in the reference's operation order,
// built without contraction so it reproduces native_relative.cpp bit for bit.
cudaError_t rel5_stage_f64(const Rel5Grid &g, const Rel5Stage &s, int blend,
                           cudaStream_t stream);

// Double storage: the exact stage with double values in a dense layout
// (g.xp == g.nx), no arrival times -- the FP64 oracle (po_rel_stage_f64 of
// the CPU restatement) on the GPU, bit for bit.  Reads s.src64 (and s.dst64
// for the blend), writes s.dst64.
cudaError_t rel5_stage_f64_storage(const Rel5Grid &g, const Rel5Stage &s, int blend,
                                   cudaStream_t stream);

// Broadcast a dense (y, x) plane of double values over every (vP, vE, psi).
cudaError_t rel5_broadcast_plane_f64(const Rel5Grid &g, const double *plane, double *field,
                                     cudaStream_t stream);

// Broadcast a (y, x) plane of initial values (dense, nx*nx) over every
// (vP, vE, psi), zero the row padding, and set arrival = start_time where the
// value is <= 0, NaN elsewhere.  With plane == nullptr the field is taken as
// already filled and only arrival (and the padding) is set.
cudaError_t rel5_init(const Rel5Grid &g, const float *plane, float *field,
                      float *arrival, float start_time, cudaStream_t stream,
                      int64_t plane_size = 0);

// Kept x range per y row for the float32 kernels: ix in [lo, hi] has
// x*x + y*y <= r2 in float32 arithmetic without contraction (x = -W + ix*dx,
// dx = 2W/(nx-1)), as the reference's float32 kernel evaluates its exit.
cudaError_t rel5_exit_rows(const Rel5Grid &g, float r2, int2 *keep, cudaStream_t stream);

// Probe values: out[i] = sum_k w[i][k] * field[idx[i][k]] in double, idx
// dense storage-order cell indices [n][32] (device arrays).
cudaError_t rel5_probe(const Rel5Grid &g, const float *field, int64_t n, const int64_t *idx,
                       const double *w, double *out, cudaStream_t stream);

// Convert one field between the padded device layout and the dense table
// layout (device to device).
cudaError_t rel5_pack(const Rel5Grid &g, const float *padded, float *dense,
                      cudaStream_t stream);
cudaError_t rel5_unpack(const Rel5Grid &g, const float *dense, float *padded,
                        cudaStream_t stream);

}  // namespace pe
