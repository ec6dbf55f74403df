/*
 * pe_b200.h — C ABI of the B200 game-value solver (libpe_b200.so).
 *
 * Plain C types only.  Every function returns PE_OK (0) or a negative error
 * code; pe_last_error() then holds a message for the calling thread.  A handle
 * owns its device buffers and one CUDA stream; the caller owns host buffers.
 * Use one handle per host thread.
 *
 * Reference interfaces these entry points replace (pursuit-evasion-core,
 * paths under src/pursuit_evasion/):
 *   - reversible/free_dp.py:259-261 runs the native executable
 *     reversible/native_relative.cpp:236-271 (argv in, fields.f32 out);
 *   - reversible/gpu_relative.py:170-179 and :322-342 launch the CuPy
 *     RawKernels `initialize` and `advance` (gpu_relative.py:26-45).
 * The relative-5D handle takes the reference executable's options
 * (native_relative.cpp:19-26, :244-262) as pe_relative_params, and performs
 * the executable's init (native_relative.cpp:91-100), its step loop
 * (:173-190) and its two stages per RK2 step (:124-172) on the GPU.
 */
#ifndef PE_B200_H
#define PE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PE_ABI_VERSION 1

enum {
  PE_OK = 0,
  PE_EINVAL = -1,     /* invalid option or argument (reference: "Invalid solver options") */
  PE_ENOMEM = -2,     /* device allocation failed */
  PE_ENONFINITE = -3, /* an update produced a non-finite value
                         (reference: native_relative.cpp:162-163) */
  PE_ETIMEOUT = -4,   /* a bounded device wait gave up */
  PE_ECUDA = -5,      /* any other CUDA runtime error */
  PE_ESTATE = -6      /* call out of order (e.g. advance before init) */
};

enum { PE_LOCAL_F32 = 0, PE_LOCAL_F64 = 1 };
enum { PE_SCHEME_ENO_LF = 0 };

/* Options of the reference executable native_relative.cpp:19-26, plus the
 * scheme, the local arithmetic precision and the CUDA device. */
typedef struct pe_relative_params {
  int32_t positions, headings, p_speeds, e_speeds; /* RelativeGrid */
  double extent;                                   /* --extent */
  double capture_radius;                           /* --radius */
  double p_speed_min, p_speed_max, p_acceleration, p_curvature;
  double e_speed_min, e_speed_max, e_acceleration, e_curvature;
  double cfl;        /* --cfl, in (0, 1] */
  int32_t order;     /* --order, 1 or 2 */
  int32_t scheme;    /* PE_SCHEME_ENO_LF */
  int32_t precision; /* PE_LOCAL_F64 reproduces the reference executable bit
                        for bit; PE_LOCAL_F32 is the fast path */
  int32_t device;    /* CUDA device ordinal */
} pe_relative_params;

typedef struct pe_relative pe_relative;

/* Library ABI version (PE_ABI_VERSION). */
int pe_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *pe_last_error(void);

/* Number of kernels this library has launched in this process. */
int64_t pe_launch_count(void);

/* Number of cells and the CFL time-step limit of a relative grid, computed
 * on the host exactly as native_relative.cpp:70-81 (no GPU needed). */
int pe_relative_cells(const pe_relative_params *params, int64_t *cells);
int pe_relative_cfl_limit(const pe_relative_params *params, double *dt_limit);

/* Validate options (native_relative.cpp:263-268) and allocate the field,
 * the stage buffer and the arrival array on params->device. */
int pe_relative_create(const pe_relative_params *params, pe_relative **out);

/* Run the handle's work on a caller-owned stream (cudaStream_t passed as
 * void*; NULL restores the handle's own stream). */
int pe_relative_set_stream(pe_relative *h, void *cuda_stream);

/* Initialise at time start_time.  initial == NULL: the circular capture field
 * float(hypot(x, y) - radius) of native_relative.cpp:91-100, computed in
 * double on the host for one (y, x) plane and broadcast on the device.
 * Otherwise a full host field of `cells` floats (a warm start or a
 * continuation).  arrival == NULL: arrival = start_time where the field is
 * <= 0, else NaN. */
int pe_relative_init(pe_relative *h, const float *initial,
                     const float *arrival, double start_time);

/* Advance the handle's time to `goal` with internal steps of
 * min(cfl_limit, goal - t) (native_relative.cpp:180-190).  Enqueues the
 * work; steps_taken (may be NULL) receives the number of steps. */
int pe_relative_advance(pe_relative *h, double goal, int64_t *steps_taken);

/* One step of exactly dt (dt > 0). */
int pe_relative_step(pe_relative *h, double dt);

/* Current time and step count. */
int pe_relative_time(const pe_relative *h, double *t, int64_t *steps);

/* Wait for the handle's work; returns PE_ENONFINITE if any update since the
 * last check produced a non-finite value. */
int pe_relative_synchronize(pe_relative *h);

/* Copy the current field / arrival times (cells floats each) to host memory
 * (synchronous; the copies come from the handle's stream). */
int pe_relative_copy_field(pe_relative *h, float *host_field);
int pe_relative_copy_arrival(pe_relative *h, float *host_arrival);

/* Initialise from a plane broadcast over the outer axes, as the reference
 * GPU path's `initialize` kernel does (gpu_relative.py:42-45, field[j] =
 * plane[j % plane_size] over the dense storage order): plane_size is
 * positions^2 (one (y, x) plane) or headings * positions^2 (a (psi, y, x)
 * block, e.g. the rectangle-contact capture field).  Arrival = start_time
 * where the value is <= 0, else NaN. */
int pe_relative_init_plane(pe_relative *h, const float *plane, int64_t plane_size,
                           double start_time);
/* Local exit (gpu_relative.py:96-101): cells with x^2 + y^2 > radius_squared
 * take the value `radius` in every stage and never arrive.  The reference
 * compiles both numbers into its kernel as literals (9 significant digits);
 * the caller passes them as it rounds them.  0, 0 disables the exit. */
int pe_relative_set_exit(pe_relative *h, double radius, double radius_squared);
/* Values of the current field at n states (gpu_relative.py:189-214,
 * :299-306): 32-corner multilinear stencils, dense storage-order cell
 * indices [n][32] and weights [n][32] (host), summed in double. */
int pe_relative_probe(pe_relative *h, int64_t n, const int64_t *indices, const double *weights,
                      double *host_out);

/* Asynchronous history output (the reference writes each output frame of
 * fields.f32 between advances with the solver stopped meanwhile,
 * native_relative.cpp:111-120).  pe_relative_snapshot packs
 * the current field into snapshot buffer `slot` (0 or 1; dense, storage
 * order) on the handle's stream and returns at once; the next advance can
 * be issued right after.  pe_relative_copy_snapshot copies that snapshot
 * to host memory on a separate copy stream once it is complete and waits
 * for the copy; it may run on another host thread while the handle
 * advances.  A slot is refilled only after its previous copy finished. */
int pe_relative_snapshot(pe_relative *h, int32_t slot);
int pe_relative_copy_snapshot(pe_relative *h, int32_t slot, float *host_field);
/* Page-locked host memory for full-speed copies (cudaHostAlloc). */
int pe_host_alloc(size_t bytes, void **out);
int pe_host_free(void *ptr);

/* Device address of the current field: storage order [vP, vE, psi, y, x]
 * with every x row padded to pe_relative_row_pitch() floats (pad = 0);
 * valid until the next step or destroy. */
int pe_relative_device_field(pe_relative *h, float **device_field);
int pe_relative_row_pitch(const pe_relative *h, int32_t *floats);

/* Tile shape of the float32 stage kernel: a CTA owns `rows` y rows of one
 * (vP, vE) pair and sweeps `psi_chunk` headings.  (0, 0) restores the
 * default; shapes that exceed the kernel's thread or shared-memory limits
 * are rejected with PE_EINVAL.  Results do not depend on the tile. */
int pe_relative_set_tile(pe_relative *h, int32_t rows, int32_t psi_chunk);
int pe_relative_get_tile(const pe_relative *h, int32_t *rows,
                         int32_t *psi_chunk);

/* Launch shape of the float32 stage kernel for the handle's tile: threads
 * per CTA, dynamic shared memory per CTA, and CTAs resident per SM at the
 * most recent launch (0 before the first). */
int pe_relative_kernel_info(const pe_relative *h, int32_t *threads,
                            int32_t *smem_bytes, int32_t *resident_ctas);

/* Sup-norm change max|V_new - V_old| of the most recent step, reduced in
 * double, and the largest increase of any cell since init (the reference's
 * maximum_increase diagnostic, native_relative.cpp:166, :233).  Synchronises. */
int pe_relative_stats(pe_relative *h, double *residual, double *max_increase);

/* Per-stage kernel timing with CUDA events on the handle's stream: enable,
 * then read the summed device milliseconds and launch count of stage 1
 * (stage=0) or stage 2 (stage=1) since enabling. */
int pe_relative_profile(pe_relative *h, int enable);
int pe_relative_kernel_time(pe_relative *h, int stage, double *total_ms,
                            int64_t *launches);

/* Release device memory and the handle. */
int pe_relative_destroy(pe_relative *h);

/* One RK2 (or RK1, params->order) step of the relative 5D ENO/LF update on
 * caller-owned device buffers, allocating no device memory.  This entry
 * point has no counterpart in the reference.  It serves callers that cannot
 * allocate once they run: a fixed-rate controller cannot afford
 * cudaMalloc/cudaFree, which may synchronise the device, and a host
 * application that owns all device memory through its own pool does not
 * allow allocations behind its back.
 *
 * field_in, field_out, arrival: device arrays of pe_relative_cells() floats
 * in the dense table layout [vP, vE, psi, y, x]; field_out receives the
 * advanced field and arrival the first-crossing times (NaN where unset).
 * t is the step's start time.  The arithmetic is the exact path, equal to a
 * PE_LOCAL_F64 handle's step bit for bit.  *residual (may be NULL) receives
 * max|field_out - field_in|.  The call synchronises `cuda_stream`.
 *
 * Scratch (the intermediate stage field, the heading tables, the reduction
 * words) lives in one fixed __device__ array of about 16.8 MB; grids above
 * PE_NOALLOC_MAX_CELLS cells or PE_NOALLOC_MAX_HEADINGS headings are
 * rejected with PE_EINVAL.  The CUDA runtime loads device code lazily, so
 * the first call on a device reserves the array there (and looks up its
 * device address); the device then holds it until the process exits.  A
 * host that gives all device memory to its own pool should make one call
 * on each device before taking the pool.  Every call copies the heading
 * tables from host memory and synchronises `cuda_stream`, so it must never
 * be called while that stream is being captured into a graph.  All calls
 * share the array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
#define PE_NOALLOC_MAX_CELLS 4194304
#define PE_NOALLOC_MAX_HEADINGS 1024
int pe_relative_step_noalloc(const pe_relative_params *params,
                             const float *field_in, float *field_out,
                             float *arrival, double t, double dt,
                             void *cuda_stream, double *residual);

/* ------------------------------------------------------------------------
 * Vehicle geometry of the compact contact game (grid construction).
 * Replaces the reference's OpenMP geometry library (local_game/
 * native_geometry.cpp:8-117 batch_clearance / batch_backups /
 * batch_actions, :221-246 configuration_connections, bound by
 * local_game/native.py:110-230 GeometryEngine).  A model is one car's
 * limits, rectangle and control period (the reference's parameter vector
 * [speed_min, speed_max, acceleration, max_curvature, length, width,
 * control_dt]); obstacles are circles [x, y, r] in a square arena of half
 * width `half_width`; states are [x, y, heading, signed speed].  Host
 * buffers in and out; the queries run one GPU thread each in double
 * precision.
 * ------------------------------------------------------------------------ */
typedef struct pe_vehicle_model {
  double speed_min, speed_max, acceleration, max_curvature;
  double length, width, control_dt;
} pe_vehicle_model;

/* Signed rectangle clearance to the walls and circles of each state. */
int pe_geometry_clearance(const pe_vehicle_model *model, const double *states, int64_t n,
                          const double *circles, int32_t n_circles, double half_width,
                          double *out, int32_t device);
/* 1 where the state is clear and one full-braking arc to rest is clear. */
int pe_geometry_backup_safe(const pe_vehicle_model *model, const double *states, int64_t n,
                            const double *circles, int32_t n_circles, double half_width,
                            uint8_t *out, int32_t device);
/* For every state and control [a, k]: next[n][na][4] the held-control arc
 * over dt, ok[n][na] = the arc is clear and its end is backup safe. */
int pe_geometry_actions(const pe_vehicle_model *model, const double *states, int64_t n,
                        const double *controls, int32_t n_controls, double dt,
                        const double *circles, int32_t n_circles, double half_width,
                        uint8_t *ok, double *next, int32_t device);
/* 1 where the straight configuration path from[i] -> to[i] is clear. */
int pe_geometry_connections(const pe_vehicle_model *model, const double *from,
                            const double *to, int64_t n, const double *circles,
                            int32_t n_circles, double half_width, uint8_t *out,
                            int32_t device);

/* ------------------------------------------------------------------------
 * FP64-storage relative 5D solve: the exact ENO/LF stage of
 * native_relative.cpp:38-172 with double values instead of float32 (the
 * reference stores float32 only; its CPU restatement with double storage is
 * the FP64 oracle po_rel_stage_f64 of oracle/relative5d.c, which this
 * reproduces bit for bit).  It exists to measure the error of
 * float32-storage tables against FP64 at sizes the CPU cannot reach.
 * Dense layout [vP, vE, psi, y, x]; initial field hypot(x, y) - r in
 * double; steps of min(cfl limit, goal - t) as pe_relative_advance; no
 * arrival times.
 * ------------------------------------------------------------------------ */
typedef struct pe_relative_f64 pe_relative_f64;

int pe_relative_f64_create(const pe_relative_params *params, pe_relative_f64 **out);
int pe_relative_f64_destroy(pe_relative_f64 *h);
int pe_relative_f64_set_stream(pe_relative_f64 *h, void *cuda_stream);
int pe_relative_f64_initialize(pe_relative_f64 *h);
int pe_relative_f64_step(pe_relative_f64 *h, double dt);
int pe_relative_f64_advance(pe_relative_f64 *h, double goal, int64_t *steps_taken);
int pe_relative_f64_time(const pe_relative_f64 *h, double *t, int64_t *steps,
                         double *cfl_dt_limit);
/* Waits; *residual = the last step's max |change|; PE_ENONFINITE if any
 * update since initialisation was not finite. */
int pe_relative_f64_stats(pe_relative_f64 *h, double *residual);
/* Waits and copies the field (pe_relative_cells doubles) to host memory. */
int pe_relative_f64_copy_field(pe_relative_f64 *h, double *host_dst);

/* ------------------------------------------------------------------------
 * vP-slab shards of one relative 5D solve (grids larger than one GPU).
 *
 * The reference solves one grid in one process (native_relative.cpp:173-190
 * step loop, run by free_dp.py:259-261); a shard runs the same stage
 * (bit-identical per cell) over global vP slabs [vp_begin, vp_end) of that
 * grid.  It holds `order` halo slabs on each side that has a neighbour
 * (the ENO stencil along vP reaches `order` slabs); after every stage the
 * caller copies the neighbours' edge slabs of the buffer just written
 * (pe_relative_shard_buffer, padded layout, slab k of the buffer at
 * (k - lo) * slab_floats floats) into those halos: peer copies or NCCL
 * send/recv on the shard's stream.  Each cell's update is the single-grid
 * stage's of the same precision (PE_LOCAL_F64 exact, PE_LOCAL_F32 fast).
 * ------------------------------------------------------------------------ */
typedef struct pe_relative_shard pe_relative_shard;

int pe_relative_shard_create(const pe_relative_params *params, int32_t vp_begin,
                             int32_t vp_end, pe_relative_shard **out);
/* slabs[4] = {lo, hi, own_lo, own_hi}: buffer slabs [lo, hi) (owned plus
 * halos) and owned slabs, global vP indices; slab_floats = padded floats
 * of one slab. */
int pe_relative_shard_layout(const pe_relative_shard *h, int32_t *slabs,
                             int64_t *slab_floats);
int pe_relative_shard_set_stream(pe_relative_shard *h, void *cuda_stream);
/* initial = NULL: the circular capture field; else the dense values of
 * buffer slabs [lo, hi) (host).  Arrival = start_time where <= 0. */
int pe_relative_shard_init(pe_relative_shard *h, const float *initial, double start_time);
/* Stage 0 (and, for order 2, stage 1) of one step of size dt; the step's
 * time advances after its last stage. */
int pe_relative_shard_stage(pe_relative_shard *h, int32_t stage, double dt);
/* The device buffer the last stage wrote (the field before any stage). */
int pe_relative_shard_buffer(const pe_relative_shard *h, float **device_buffer);
/* Owned slabs of the field / arrival, dense, to host. */
int pe_relative_shard_copy_field(pe_relative_shard *h, float *host_owned);
int pe_relative_shard_copy_arrival(pe_relative_shard *h, float *host_owned);
/* Sup-norm change of the owned cells in the last step, and the largest
 * increase; combine over shards with a maximum. */
int pe_relative_shard_stats(pe_relative_shard *h, double *residual, double *increase);
int pe_relative_shard_synchronize(pe_relative_shard *h);
int pe_relative_shard_destroy(pe_relative_shard *h);

/* ------------------------------------------------------------------------
 * Batched relative 5D solves.
 *
 * Many independent free_dp-style solves -- each with its own RelativeGrid,
 * physics and horizon -- advanced together: every RK2 step of every solve
 * runs in ONE persistent cooperative kernel launch (recorded once in a
 * CUDA graph), a grid-wide barrier between stages.  Each solve follows the
 * reference executable's driver (native_relative.cpp:173-190, steps of
 * min(cfl_limit, horizon - t)) from the capture field
 * (native_relative.cpp:91-100); with the exact arithmetic its final field
 * and arrival times equal a PE_LOCAL_F64 pe_relative handle's (and the
 * reference executable's run with the same --horizon and --output-dt =
 * horizon) bit for bit.  The reference has no batched mode: it runs such
 * solves one executable at a time (free_dp.py:259-261).
 * ------------------------------------------------------------------------ */
typedef struct pe_batch pe_batch;

/* params[i].order must be 2 and every solve must have the same precision:
 * PE_LOCAL_F64 (the exact arithmetic, bit-identical per solve as above) or
 * PE_LOCAL_F32 (a float32 cell update, within float rounding and ENO
 * selection ties of the exact one).  params[i].device is ignored (the batch
 * lives on `device`). */
int pe_batch_create(const pe_relative_params *params, const double *horizons,
                    int32_t count, int32_t device, pe_batch **out);
/* Work-item tile of one solve: `rows` y rows of one (vP, vE, psi) plane.
 * Results do not depend on the tile. */
int pe_batch_set_tile(pe_batch *h, int32_t solve, int32_t rows);
int pe_batch_get_tile(const pe_batch *h, int32_t solve, int32_t *rows);
int pe_batch_set_stream(pe_batch *h, void *cuda_stream);
/* Capture field and arrival of every solve at t = 0. */
int pe_batch_init(pe_batch *h);
/* All steps of all solves: one graph launch holding one cooperative kernel.
 * Enqueues the work; init must precede every run. */
int pe_batch_run(pe_batch *h);
/* Wait; PE_ETIMEOUT if a barrier wait gave up, PE_ENONFINITE if any update
 * was not finite. */
int pe_batch_synchronize(pe_batch *h);
/* Cells, RK2 steps to the horizon and the CFL step limit of one solve. */
int pe_batch_solve_info(const pe_batch *h, int32_t solve, int64_t *cells,
                        int64_t *steps, double *dt_limit);
/* Dense [vP, vE, psi, y, x] field / arrival times of one solve (host). */
int pe_batch_copy_field(pe_batch *h, int32_t solve, float *host_field);
int pe_batch_copy_arrival(pe_batch *h, int32_t solve, float *host_arrival);
/* Sup-norm change of the solve's last step and its largest increase. */
int pe_batch_stats(pe_batch *h, int32_t solve, double *residual,
                   double *max_increase);
/* CTAs and threads of the persistent launch, the longest solve's steps and
 * the batch's cell-stage updates per run (2 x cells x steps, summed). */
int pe_batch_launch_info(const pe_batch *h, int32_t *ctas, int32_t *threads,
                         int32_t *max_steps, int64_t *total_cell_stages);
int pe_batch_profile(pe_batch *h, int enable);
int pe_batch_kernel_time(pe_batch *h, double *total_ms, int64_t *launches);
int pe_batch_destroy(pe_batch *h);

/* ------------------------------------------------------------------------
 * Dense 8D game [xP, yP, thP, vP, xE, yE, thE, vE] (vE fastest).
 *
 * Replaces the reference executable native_world.cpp (argv options
 * :76-110, surfaces :155-176, stage :261-314, frame loop :315-336) run by
 * reversible/world_dp.py:361-372, and the CuPy kernels `init`/`advance` of
 * reversible/gpu_map_game.py:43-75 (without obstacle clearance grids).
 * Arithmetic is float32 in the reference's order and reproduces the
 * executable bit for bit.
 * ------------------------------------------------------------------------ */
typedef struct pe_world_params {
  int32_t positions, headings, p_speeds, e_speeds; /* WorldGrid */
  double extent;         /* --extent */
  double arena;          /* --arena (square half width; avoid_mode 1) */
  double capture_radius; /* --radius (square surfaces init) */
  double p_speed_min, p_speed_max, p_acceleration, p_curvature;
  double e_speed_min, e_speed_max, e_acceleration, e_curvature;
  double cfl;                    /* --cfl */
  int32_t order;                 /* --order, 1 or 2 */
  int32_t linear_speed_boundary; /* --linear-speed-boundary */
  int32_t avoid_mode;            /* 0: none; 1: max(|xP|,|yP|) - arena + 1e-6;
                                    2: -p_clear[xP, yP, thP] + 1e-6 (obstacle map,
                                    gpu_map_game.py:64-66; pe_world_set_clearance) */
  int32_t device;
  int32_t fast; /* 0 (default): float32 in the reference's order, bit for bit
                   native_world.cpp; 1: reciprocal spacings and multiply-add
                   contraction (equal to float rounding and ENO2 flips) */
} pe_world_params;

typedef struct pe_world pe_world;

int pe_world_cells(const pe_world_params *params, int64_t *cells);
/* dt bound of native_world.cpp:133-135. */
int pe_world_dt_limit(const pe_world_params *params, double *dt);
int pe_world_create(const pe_world_params *params, pe_world **out);
/* Capture field: oriented-rectangle contact value (separating axes, double,
 * local_game/geometry.py:15-36) of the two footprints at every grid pose;
 * arrival 0 where <= 0. */
int pe_world_init_contact(pe_world *h, double p_length, double p_width,
                          double e_length, double e_width);
/* The reference's square-arena surfaces (native_world.cpp:155-176). */
int pe_world_init_square(pe_world *h);
/* Obstacle map game (gpu_map_game.py:45-50, :64-66): each car's clearance
 * per (x, y, heading) pose, positions^2 * headings floats in C order
 * [x][y][heading] (host), as FootprintMap.clearance gives them
 * (gpu_map_game.py:78-84).  Avoid mode 2 floors every update at
 * -p_clear + 1e-6. */
int pe_world_set_clearance(pe_world *h, const float *p_clear, const float *e_clear);
/* Surfaces of the map game: max(min(hypot(dP - dE) - radius, e_clear),
 * -p_clear + 1e-6); arrival 0 where <= 0. */
int pe_world_init_map(pe_world *h);
/* A host field (continuation, native_world.cpp:177-191). */
int pe_world_init_field(pe_world *h, const float *field, const float *arrival,
                        double start_time);
int pe_world_advance(pe_world *h, double goal, int64_t *steps_taken);
int pe_world_step(pe_world *h, double dt);
int pe_world_time(const pe_world *h, double *t, int64_t *steps);
int pe_world_synchronize(pe_world *h);
int pe_world_copy_field(pe_world *h, float *host_field);
int pe_world_copy_arrival(pe_world *h, float *host_arrival);
/* max |V_new - V_old| of the most recent step. */
int pe_world_residual(pe_world *h, double *residual);
int pe_world_set_stream(pe_world *h, void *cuda_stream);
int pe_world_profile(pe_world *h, int enable);
int pe_world_kernel_time(pe_world *h, double *total_ms, int64_t *launches);
int pe_world_destroy(pe_world *h);

/* ------------------------------------------------------------------------
 * Relative 5D semi-Lagrangian min-max backup.
 *
 * No reference counterpart computes this 5D backup; it composes the
 * reference's held-command successor (reversible/model.py:86-183), action
 * catalogue (reversible/controllers.py:19-27), min-P/max-E order with the
 * tube minimum (local_game/grid_game.py:218-230, the CUDA kernels
 * `interpolate_p`/`reduce_e` it replaces in spirit) and 5D multilinear
 * stencil (reversible/relative_table.py:76-102).
 * ------------------------------------------------------------------------ */
enum { PE_SL_TUBE = 0, PE_SL_MINTIME = 1 };

typedef struct pe_semilag_params {
  int32_t positions, headings, p_speeds, e_speeds; /* RelativeGrid */
  double extent, capture_radius;
  double p_speed_min, p_speed_max, p_acceleration, p_curvature;
  double e_speed_min, e_speed_max, e_acceleration, e_curvature;
  double dt;     /* held-command step; 0 selects the interpolation CFL step
                    (no coordinate moves more than one grid spacing) */
  int32_t mode;  /* PE_SL_TUBE: V' = min(V, min_u max_w V(s'));
                    PE_SL_MINTIME: u' = 0 in the capture disk, else
                    (1 - e^-dt) + e^-dt * min_u max_w u(s'), u = 1 - e^-T */
  int32_t device;
} pe_semilag_params;

typedef struct pe_semilag pe_semilag;

int pe_semilag_dt(const pe_semilag_params *params, double *dt);
int pe_semilag_create(const pe_semilag_params *params, pe_semilag **out);
/* initial == NULL: TUBE hypot(x,y) - r; MINTIME 0 in the capture disk, 1
 * elsewhere.  Otherwise a dense host field (a warm start). */
int pe_semilag_init(pe_semilag *h, const float *initial);
/* Initialise from a dense field already on the handle's device (e.g. the
 * learned surrogate's prediction). */
int pe_semilag_init_device(pe_semilag *h, const float *device_initial);
/* One backup sweep; with_policy != 0 also records the optimal pursuer and
 * evader action indices (catalogue order 3*i_a + i_k) of every cell. */
int pe_semilag_backup(pe_semilag *h, int with_policy);
/* Value iteration: up to max_iterations backups, checking the sup-norm
 * change every check_every sweeps; stops once it is below tol (tol = 0: run
 * all sweeps). */
int pe_semilag_iterate(pe_semilag *h, int64_t max_iterations, double tol,
                       int32_t check_every, int64_t *iterations,
                       double *residual, int32_t *converged);
int pe_semilag_residual(pe_semilag *h, double *residual);
/* Waits; action-pair evaluations (one interpolated successor value each)
 * of the tiled value backups since the last pe_semilag_init*: the probes,
 * full reply scans and pruned replies of every live cell.  Divided by the
 * cells and backups it is the work per cell behind the backup's on-chip
 * rate; the generic kernel does not count (0). */
int pe_semilag_evaluations(pe_semilag *h, int64_t *evaluations);
/* Work skipping of the tiled value backups (on by default): a work item
 * (one speed pair and y tile over all headings) whose neighbouring items
 * (speed pairs and tiles +-1, the reach of every successor) left all their
 * cells unchanged, bit for bit, in the previous backup reads the same
 * inputs as then, so its cells are copied instead of recomputed.  Results
 * are identical with and without it.  No counterpart in the reference. */
int pe_semilag_set_skip(pe_semilag *h, int enable);
/* Waits; work items of the tiled kernel computed (not skipped) since the
 * last pe_semilag_init*. */
int pe_semilag_items_computed(pe_semilag *h, int64_t *items);
int pe_semilag_copy_value(pe_semilag *h, float *host_value);
/* Copy the value field into a dense device array on the handle's device. */
int pe_semilag_copy_value_device(pe_semilag *h, float *device_value);
int pe_semilag_copy_policy(pe_semilag *h, uint8_t *host_p, uint8_t *host_e);
int pe_semilag_device_value(pe_semilag *h, float **device_value);
int pe_semilag_iterations(const pe_semilag *h, int64_t *iterations);
int pe_semilag_set_stream(pe_semilag *h, void *cuda_stream);
/* Kernel of value-only backups.  PE_SL_KERNEL_TILED stages speed-blended
 * heading planes of a tile in shared memory and prunes pursuer actions
 * (needs positions + 4 <= 72 and successors within 1.99 cells and one
 * heading plane, true at the interpolation-CFL dt); PE_SL_KERNEL_GENERIC
 * gathers from global memory; PE_SL_KERNEL_AUTO (default) picks the tiled
 * kernel where it applies and the grid gives at least 8 of its work items
 * ((vP, vE) pairs x row tiles) per SM.  Backups that record the policy always use the
 * generic kernel.  Both give the same values up to float rounding. */
enum { PE_SL_KERNEL_AUTO = 0, PE_SL_KERNEL_GENERIC = 1, PE_SL_KERNEL_TILED = 2 };
int pe_semilag_set_kernel(pe_semilag *h, int kernel);
/* Tile of the tiled kernel: about `rows` cell rows at full width per work
 * item (0 restores the default); smaller tiles use less shared memory, so
 * two CTAs can share an SM, at a larger halo cost.  Results do not depend
 * on the tile. */
int pe_semilag_set_tile(pe_semilag *h, int32_t rows);
int pe_semilag_get_tile(const pe_semilag *h, int32_t *rows, int32_t *threads,
                        int64_t *items);
/* The kernel value-only backups use now (GENERIC or TILED). */
int pe_semilag_kernel(const pe_semilag *h, int32_t *kernel);
int pe_semilag_profile(pe_semilag *h, int enable);
int pe_semilag_kernel_time(pe_semilag *h, double *total_ms, int64_t *launches);
/* Arrival times of the tube field (PE_SL_TUBE only), as the ENO/LF path
 * keeps them (native_relative.cpp:167-168): after every backup from the
 * start time t, a cell whose value went from > 0 to <= 0 for the first time
 * gets t + dt * prev / (prev - value).  host_arrival != NULL continues an
 * earlier record (N floats, NaN = not arrived); NULL starts one: start_time
 * where the current value is <= 0, NaN elsewhere. */
int pe_semilag_track_arrival(pe_semilag *h, const float *host_arrival, double start_time);
int pe_semilag_copy_arrival(pe_semilag *h, float *host_arrival);
int pe_semilag_destroy(pe_semilag *h);

/* ------------------------------------------------------------------------
 * Learned value surrogate: BF16 tensor-core MLP kernels.
 *
 * The reference has no learned warm start for the game tables; the closest
 * precedent is its SiLU MLP value heads trained by supervised MSE on DP
 * labels with Adam(W) (pe/local_game/learning.py:14-77 ContactValueNet,
 * pe/local_game/training.py:39 fit_contact_values, :185-186 optimiser,
 * :352 loss).  These building blocks run a features -> 4 x 256 SiLU -> 1
 * network in BF16 with FP32 accumulation and FP32 master weights; the host
 * side (pursuit_evasion_b200/learned) chains them into training steps that
 * are captured in one CUDA graph.  Every pointer is a device pointer; bf16
 * arrays are passed as void*.  All calls are asynchronous on cuda_stream.
 * ------------------------------------------------------------------------ */

/* C = A x B.  a_mmajor: A stored [K][M] (else [M][K]); b_nmajor: B stored
 * [K][N] (else [N][K]).  epilogue 0: C32 = acc; 1: C32 = acc + bias (C32 may
 * be NULL), C16 = bf16(silu(acc + bias)); 2: C32 += acc, split-K over
 * `splits` CTAs (C32 pre-zeroed); 3: C16 = bf16(acc * silu'(zpre)).
 * M, N multiples of 128, K a multiple of 32 * splits. */
int pe_mlp_gemm(const void *A, const void *B, int M, int N, int K, int lda, int ldb,
                int a_mmajor, int b_nmajor, int epilogue, int splits, float *C32,
                void *C16, int ldc, const float *bias, const float *zpre,
                void *cuda_stream);
/* The same product on the 5th-generation tensor cores (tcgen05.mma with the
 * accumulator in tensor memory, TMA-fed 128B-swizzled shared memory), for
 * the case of both operands K-major: A [M][K] (row pitch lda) and B [N][K]
 * (row pitch ldb), C = A B^T.  Epilogues 0, 1 and 3 as pe_mlp_gemm.  M, N
 * multiples of 128, K a multiple of 64, operands 16-byte aligned with lda,
 * ldb multiples of 8. */
int pe_mlp_gemm_tc(const void *A, const void *B, int M, int N, int K, int lda, int ldb,
                   int epilogue, float *C32, void *C16, int ldc, const float *bias,
                   const float *zpre, void *cuda_stream);
/* C32 += A B^T on the tensor cores with split-K: both operands K-major as
 * pe_mlp_gemm_tc, the K range cut into `splits` equal parts, one CTA per
 * 128 x 128 tile and part, each adding its partial tile to C32 with 16-byte
 * FP32 atomics (C32 pre-zeroed by the caller; the summation order, and so
 * the last bits, vary between runs).  The weight gradients of the
 * surrogate: A = transposed activation gradients [out][rows], B =
 * transposed layer inputs [in][rows], K = rows.  M, N multiples of 128, K a
 * multiple of 64 * splits; A, B, C32 16-byte aligned; lda, ldb >= K
 * multiples of 8; ldc >= N a multiple of 4. */
int pe_mlp_gemm_tc_splitk(const void *A, const void *B, int M, int N, int K, int lda, int ldb,
                          int splits, float *C32, int ldc, void *cuda_stream);
/* Number of pe_mlp_gemm_tc launches whose bounded waits timed out since the
 * last call (then cleared).  Synchronises the device. */
int pe_mlp_gemm_tc_timeouts(int32_t *count);
/* Adam on n FP32 master weights w (w16, if not NULL, receives their bf16
 * copy).  corr[0], corr[1] are the bias corrections 1 - beta^t read on the
 * device, so a captured graph replays with the current step. */
int pe_mlp_adam(float *w, void *w16, const float *grad, float *m, float *v, int64_t n,
                float lr, float beta1, float beta2, float eps, const float *corr,
                float grad_scale, void *cuda_stream);
/* Output head y = h . w + b over bf16 activations h [rows][width]; with a
 * target also dy = 2 (y - target) / rows and loss += mean squared error. */
int pe_mlp_head_forward(const void *h, const float *w, const float *b,
                        const float *target, float *y, float *dy, float *loss,
                        int rows, int width, void *cuda_stream);
/* Head gradients dw, db and dz = dy w * silu'(zprev) (bf16) for the last
 * hidden layer. */
int pe_mlp_head_backward(const void *h, const float *zprev, const float *w,
                         const float *dy, float *dw, float *db, void *dz, int rows,
                         int width, void *cuda_stream);
/* dst[c][r] = src[r][c] for a bf16 matrix of rows x cols (the transposed
 * weight copy the tensor-core activation-gradient GEMM reads). */
int pe_mlp_transpose(const void *src, void *dst, int rows, int cols, void *cuda_stream);
/* out[c] = sum over rows of bf16 x[row][c] (bias gradients). */
int pe_mlp_colsum(const void *x, float *out, int rows, int cols, void *cuda_stream);
/* Features of relative 5D grid nodes (flat [vP, vE, psi, y, x] indices idx)
 * into bf16 rows of width ld (x, y, cos psi, sin psi, vP, vE scaled to
 * [-1, 1]); with a table also target[i] = table[idx[i]]. */
int pe_mlp_encode_relative_nodes(const float *table, const int64_t *idx, int n,
                                 int positions, int headings, int p_speeds,
                                 int e_speeds, double extent, double p_min,
                                 double p_max, double e_min, double e_max, void *feat,
                                 int ld, float *target, void *cuda_stream);
/* Features of arbitrary relative states [n][5] = (x, y, psi, vP, vE). */
int pe_mlp_encode_relative_states(const float *states, int n, double extent,
                                  double p_min, double p_max, double e_min,
                                  double e_max, void *feat, int ld, void *cuda_stream);
/* Features of 8D grid nodes [xP, yP, thP, vP, xE, yE, thE, vE] (10 columns:
 * positions, cos/sin of both headings, both speeds). */
int pe_mlp_encode_world_nodes(const float *table, const int64_t *idx, int n,
                              int positions, int headings, int p_speeds, int e_speeds,
                              double extent, double p_min, double p_max, double e_min,
                              double e_max, void *feat, int ld, float *target,
                              void *cuda_stream);

/* ------------------------------------------------------------------------
 * Queries of a completed relative table, resident on the GPU.
 *
 * Replaces RelativeTable.field / RelativeTable.value of
 * reversible/relative_table.py:76-161 for batches of states: 32-corner
 * multilinear stencil over [vP, vE, psi, y, x] with periodic heading, the
 * signed field at a budget (linear in time between frames), and the capture
 * time as the first zero crossing found by bisection over frames.  Results
 * equal the reference reader's in double precision (summation order
 * aside), including its batch-wide bisection: a state whose earliest frame
 * is already inside is resolved as the reference resolves it in a batch
 * of the same states.
 * ------------------------------------------------------------------------ */
typedef struct pe_table pe_table;

/* host_frames: [frames][cells] float32 in storage order [vP, vE, psi, y, x]
 * (fields.f32 of a table directory); times: the output times; shape,
 * axis_lo, axis_hi, spacing per storage axis (the metadata's axes: first,
 * last and second-minus-first value); speed_limits = {vP min, vP max, vE
 * min, vE max}. */
int pe_table_create(const float *host_frames, int32_t frames, const double *times,
                    const int32_t shape[5], const double axis_lo[5], const double axis_hi[5],
                    const double spacing[5], double capture_radius,
                    const double speed_limits[4], int32_t device, pe_table **out);
/* Capture times of n states [n][5] = (x, y, psi, vP, vE) (host arrays). */
int pe_table_value(pe_table *h, const double *host_states, int64_t n, double *host_out);
/* Signed field of n states at budgets[n] (host arrays). */
int pe_table_field(pe_table *h, const double *host_states, const double *host_budgets,
                   int64_t n, double *host_out);
int pe_table_destroy(pe_table *h);

/* ------------------------------------------------------------------------
 * Legacy six-dimensional square game [xP, yP, thP, xE, yE, thE] with
 * constant speeds and bounded turn rates.
 *
 * Replaces the executable src/pursuit_evasion/dp/native_square.cpp (argv
 * in, fields.f32 out), run by dp/native.py:14-106.  The options are its
 * argv (native_square.cpp:65-80); init is its target/avoid surfaces
 * (:110-128), advance its frame loop (:185-198) and the stage its ENO1/ENO2
 * LF RK1/RK2 update (:145-183), in float32 in the reference's operation
 * order: fields equal the executable's bit for bit.
 * ------------------------------------------------------------------------ */
typedef struct pe_square_params {
  int32_t positions, headings;     /* --positions, --headings */
  double extent, arena;            /* --extent (> arena), --arena */
  double capture_radius;           /* --radius */
  double p_speed, e_speed;         /* --vp, --ve */
  double p_turn_rate, e_turn_rate; /* --wp, --we */
  double cfl;                      /* --cfl, in (0, 1] */
  int32_t order;                   /* --order, 1 or 2 */
  int32_t device;                  /* CUDA device ordinal */
} pe_square_params;

typedef struct pe_square pe_square;

int pe_square_cells(const pe_square_params *params, int64_t *cells);
/* max_internal_dt of native_square.cpp:94-95 (host only). */
int pe_square_dt_limit(const pe_square_params *params, double *dt);
int pe_square_create(const pe_square_params *params, pe_square **out);
/* max(target, avoid) and arrival (0 where <= 0, else NaN); time 0. */
int pe_square_init(pe_square *h);
/* Internal steps of min(dt_limit, goal - t) until t >= goal - 1e-10. */
int pe_square_advance(pe_square *h, double goal, int64_t *steps_taken);
int pe_square_time(const pe_square *h, double *t, int64_t *steps);
int pe_square_synchronize(pe_square *h);
int pe_square_copy_field(pe_square *h, float *host_field);
int pe_square_copy_arrival(pe_square *h, float *host_arrival);
/* Sup-norm change of the last step (synchronises). */
int pe_square_residual(pe_square *h, double *residual);
int pe_square_profile(pe_square *h, int32_t enable);
int pe_square_kernel_time(pe_square *h, double *total_ms, int64_t *launches);
int pe_square_destroy(pe_square *h);

/* ------------------------------------------------------------------------
 * Compact eight-state semi-Lagrangian contact game (local pair game).
 *
 * Replaces the CuPy RawKernels and host loops of
 * src/pursuit_evasion/local_game/grid_game.py:
 *   gpu_arrays / initialize_gpu / backup_gpu            :226-333 (dense)
 *   packed_gpu_arrays / initialize_packed / backup_packed :424-581 (pairs
 *                                                        within the exit radius)
 * and the packed query of local_game/reference.py:122-134 (query_field).
 *
 * Each car has n legal four-dimensional states (x, y, heading, speed) and
 * n_actions held controls; a control's successor is a 16-vertex
 * interpolation stencil (ids, weights) over the car's own states.  One
 * backup sets, for every pair (ip, ie) of the domain,
 *   V'(ip, ie) = min(V, min_{u allowed} max_{a allowed}
 *                sum_q we[q] sum_k wp[k] V(idp[k], ide[q]))
 * (the reference's factorized product interpolation; its early exit
 * `worst >= best` is kept).  The dense layout is [n_p][n_e]; pairs farther
 * apart than the exit radius keep their value.  The packed layout stores
 * only the domain's pairs (PairDomain, grid_game.py:336-381); a vertex
 * outside the domain, or an evader state beyond the pursuer's reach, reads
 * the exit value.  Unlike the reference, one launch performs a whole backup
 * with the field resident on the device (no per-chunk launches, no host
 * round trip of the output tiles).
 * ------------------------------------------------------------------------ */
typedef struct pe_compact pe_compact;

/* One car's grid (VehicleGrid, grid_game.py:21-30); host arrays, copied. */
typedef struct pe_vehicle_grid {
  int32_t states;          /* n */
  int32_t actions;         /* n_actions */
  const float *pose;       /* [n][4] x, y, heading, speed */
  const int32_t *ids;      /* [n][n_actions][16] successor vertex ids */
  const float *weights;    /* [n][n_actions][16] vertex weights (<= 0: unused) */
  const uint8_t *allowed;  /* [n][n_actions] */
} pe_vehicle_grid;

/* PairDomain (grid_game.py:336-381); host arrays, copied. */
typedef struct pe_pair_domain {
  int32_t positions;         /* distinct pursuer positions */
  int32_t max_count;         /* row length of e_indices */
  const int32_t *p_position; /* [n_p] position index of each pursuer state */
  const int32_t *lookup;     /* [positions][n_e] rank of an evader state, -1 outside */
  const int32_t *e_indices;  /* [positions][max_count] evader states in range */
  const int32_t *counts;     /* [positions] */
  const int64_t *offsets;    /* [n_p + 1] first pair of each pursuer state */
} pe_pair_domain;

/* domain == NULL: dense layout.  exit_radius: the domain's radius (packed)
 * or the capture field's exit radius (dense). */
int pe_compact_create(const pe_vehicle_grid *p, const pe_vehicle_grid *e,
                      const pe_pair_domain *domain, double exit_radius,
                      int32_t device, pe_compact **out);
/* Number of stored pairs (n_p * n_e dense, offsets[n_p] packed). */
int pe_compact_cells(const pe_compact *h, int64_t *out);
/* Capture field: oriented-rectangle separation of the two footprints in
 * float32 (grid_game.py:193-201 / :364-372); dense pairs beyond the exit
 * radius get the exit radius. */
int pe_compact_init(pe_compact *h, double p_length, double p_width, double e_length,
                    double e_width);
int pe_compact_set_field(pe_compact *h, const float *host, int64_t n);
/* `count` backups, each one kernel launch on the handle's stream. */
int pe_compact_backup(pe_compact *h, int32_t count);
int pe_compact_copy_field(pe_compact *h, float *host, int64_t n);
/* Device pointer of the current field (valid until the next backup). */
int pe_compact_field_device(pe_compact *h, void **out);
/* n queries, each a product of a pursuer and an evader 16-vertex stencil
 * (host arrays [n][16]); packed handles read the exit value outside the
 * domain (reference.py:122-134). */
int pe_compact_query(pe_compact *h, int32_t n, const int32_t *p_ids,
                     const float *p_weights, const int32_t *e_ids,
                     const float *e_weights, float *host_out);
int pe_compact_set_stream(pe_compact *h, void *cuda_stream);
int pe_compact_synchronize(pe_compact *h);
/* Device time of the backups since profiling was switched on. */
int pe_compact_profile(pe_compact *h, int32_t enable);
int pe_compact_kernel_time(pe_compact *h, double *ms, int64_t *launches);
int pe_compact_destroy(pe_compact *h);

#ifdef __cplusplus
}
#endif
#endif /* PE_B200_H */
