// pe_relative_step_noalloc: one relative 5D ENO/LF step on caller-owned
// device buffers, without any device allocation.
//
// Some callers cannot allocate device memory once they are running: a
// fixed-rate pursuit controller must not stall on cudaMalloc/cudaFree
// (either may synchronise the whole device), and a host application that
// hands all device memory out of its own pool does not let plugins allocate
// behind its back.  For them this entry point keeps its scratch -- the RK2
// intermediate stage field, the heading sine/cosine tables and the
// reduction words -- in one file-scope __device__ array of fixed size,
// which every GPU that uses this entry point holds until the process exits.
// The CUDA runtime loads a library's device code lazily (per translation
// unit, on first use), so the array is reserved on a device by the first
// call there, not when the library is loaded: a host that hands all device
// memory to its own pool makes one call first (any small grid will do).
//
// The caller passes the field to advance, the field to write and the
// arrival times, all in the dense table layout [vP, vE, psi, y, x].  The
// arithmetic is the exact path (double local, native_relative.cpp order),
// so the result equals pe_relative_step on a PE_LOCAL_F64 handle bit for
// bit.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "pe_internal.h"
#include "relative5d.cuh"

namespace {

// Scratch layout (in doubles): stats words, sin table, cos table, then the
// stage field (floats).  Headings are limited to PE_NOALLOC_MAX_HEADINGS.
constexpr int kMaxHeadings = PE_NOALLOC_MAX_HEADINGS;
constexpr size_t kStatsDoubles = 4;  // pe::Rel5Stats is 24 bytes
constexpr size_t kStageOffsetDoubles = kStatsDoubles + 2 * kMaxHeadings;
constexpr size_t kScratchDoubles =
    kStageOffsetDoubles + (size_t)PE_NOALLOC_MAX_CELLS / 2;

static __device__ __align__(256) double g_step_scratch[kScratchDoubles];

static_assert(sizeof(pe::Rel5Stats) <= kStatsDoubles * sizeof(double),
              "reduction words must fit their scratch slot");

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device; the symbol's host-side name is not a device address).
int scratch_address(int device, double **out) {
  if (device < 0 || device >= kMaxDevices)
    return pe::fail(PE_EINVAL, "device ordinal %d out of range", device);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void *ptr = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&ptr, g_step_scratch);
    if (err != cudaSuccess) return pe::cuda_fail(err, "cudaGetSymbolAddress(scratch)");
    g_scratch_ptr[device] = static_cast<double *>(ptr);
  }
  *out = g_scratch_ptr[device];
  return PE_OK;
}

}  // namespace

extern "C" int pe_relative_step_noalloc(const pe_relative_params *params,
                                        const float *field_in, float *field_out,
                                        float *arrival, double t, double dt,
                                        void *cuda_stream, double *residual) {
  using pe::fail;
  if (!params) return fail(PE_EINVAL, "params is NULL");
  if (!field_in || !field_out || !arrival)
    return fail(PE_EINVAL, "field_in, field_out and arrival are required");
  if (field_in == field_out) return fail(PE_EINVAL, "field_in and field_out must differ");
  if (!(dt > 0) || !std::isfinite(dt) || !std::isfinite(t))
    return fail(PE_EINVAL, "t must be finite and dt > 0");
  int64_t cells = 0;
  int rc = pe_relative_cells(params, &cells);  // validates the options
  if (rc) return rc;
  if (cells > (int64_t)PE_NOALLOC_MAX_CELLS)
    return fail(PE_EINVAL,
                "grid has %lld cells; pe_relative_step_noalloc handles at most %d",
                (long long)cells, PE_NOALLOC_MAX_CELLS);
  if (params->headings > kMaxHeadings)
    return fail(PE_EINVAL, "at most %d headings without allocation", kMaxHeadings);
  PE_CUDA_TRY(cudaSetDevice(params->device));
  double *scratch = nullptr;
  rc = scratch_address(params->device, &scratch);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);

  // Dense grid: the exact kernel addresses cells through strides, so the
  // table layout is used as it is (no row padding).
  const double pi = std::acos(-1.0);
  pe::Rel5Grid g{};
  g.nx = params->positions;
  g.nh = params->headings;
  g.nvp = params->p_speeds;
  g.nve = params->e_speeds;
  g.order = params->order;
  g.xp = g.nx;
  g.sy = g.nx;
  g.sp = (int64_t)g.nx * g.nx;
  g.se = g.sp * g.nh;
  g.sv = g.se * g.nve;
  g.n = g.n_padded = g.sv * g.nvp;
  g.extent = params->extent;
  g.dx = 2 * params->extent / (params->positions - 1);
  g.dphi = 2 * pi / params->headings;
  g.dvp = (params->p_speed_max - params->p_speed_min) / (params->p_speeds - 1);
  g.dve = (params->e_speed_max - params->e_speed_min) / (params->e_speeds - 1);
  g.vp_lo = params->p_speed_min;
  g.ve_lo = params->e_speed_min;
  g.acc_p = params->p_acceleration;
  g.acc_e = params->e_acceleration;
  g.curv_p = params->p_curvature;
  g.curv_e = params->e_curvature;
  pe::set_reciprocals(g);

  // Heading tables (native_relative.cpp:84-89) into the scratch array:
  // only the nh sines and nh cosines this grid uses are copied.
  double sines[kMaxHeadings], cosines[kMaxHeadings];
  for (int k = 0; k < g.nh; k++) {
    const double q = -pi + k * g.dphi;
    sines[k] = std::sin(q);
    cosines[k] = std::cos(q);
  }
  pe::Rel5Stats *stats = reinterpret_cast<pe::Rel5Stats *>(scratch);
  double *sn = scratch + kStatsDoubles;
  double *cs = sn + kMaxHeadings;
  float *stage = reinterpret_cast<float *>(scratch + kStageOffsetDoubles);
  PE_CUDA_TRY(cudaMemsetAsync(stats, 0, sizeof(pe::Rel5Stats), stream));
  PE_CUDA_TRY(cudaMemcpyAsync(sn, sines, sizeof(double) * g.nh, cudaMemcpyHostToDevice,
                              stream));
  PE_CUDA_TRY(cudaMemcpyAsync(cs, cosines, sizeof(double) * g.nh, cudaMemcpyHostToDevice,
                              stream));

  pe::Rel5Stage s{};
  s.arrival = arrival;
  s.sn = sn;
  s.cs = cs;
  s.dt = dt;
  s.t = t;
  s.stats = stats;
  if (g.order == 1) {
    s.src = field_in;
    s.dst = field_out;
    PE_CUDA_TRY(pe::rel5_stage_f64(g, s, 0, stream));
    pe::count_launches(1);
  } else {
    // Stage 2 averages with the old value read from its output buffer.
    PE_CUDA_TRY(cudaMemcpyAsync(field_out, field_in, sizeof(float) * (size_t)cells,
                                cudaMemcpyDeviceToDevice, stream));
    s.src = field_in;
    s.dst = stage;
    PE_CUDA_TRY(pe::rel5_stage_f64(g, s, 0, stream));
    s.src = stage;
    s.dst = field_out;
    PE_CUDA_TRY(pe::rel5_stage_f64(g, s, 1, stream));
    pe::count_launches(2);
  }
  pe::Rel5Stats host{};
  PE_CUDA_TRY(cudaMemcpyAsync(&host, stats, sizeof host, cudaMemcpyDeviceToHost, stream));
  PE_CUDA_TRY(cudaStreamSynchronize(stream));
  if (host.timeout) return fail(PE_ETIMEOUT, "a bounded device wait gave up");
  if (host.nonfinite) return fail(PE_ENONFINITE, "Nonfinite field update");
  if (residual) std::memcpy(residual, &host.residual, sizeof(double));
  return PE_OK;
}
