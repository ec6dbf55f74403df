// C-ABI of one vP-slab shard of the relative 5D solve (declared in
// include/pe_b200.h, pe_relative_shard_*).
//
// The storage order [vP, vE, psi, y, x] makes each vP index one contiguous
// slab of nve * nh * nx * xp floats.  A shard owns global slabs
// [own_lo, own_hi) and keeps `order` halo slabs on each side that has a
// neighbour: the ENO stencil along vP reads at most `order` slabs away.
// Stages run the exact kernel (relative5d_exact.cu) or the float32 kernel
// (relative5d_fast.cu) over the owned slabs only, with global vP indices,
// so the speed boundary rule and the vP values are those of the whole grid.
// After each stage the caller refreshes the halo slabs of the buffer just
// written from the neighbouring shards (peer copies, NCCL send/recv); the
// handle only exposes that buffer.
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "pe_internal.h"
#include "relative5d.cuh"
#include "relative5d_host.h"

struct pe_relative_shard {
  pe_relative_params p{};
  pe::Rel5Grid g{};  // global geometry; own_lo / own_n / slab_lo set
  pe::Rel5Tile tile{};  // float32 stage tiling
  int lo = 0, hi = 0, own_lo = 0, own_hi = 0;
  double t = 0;
  int64_t steps = 0;
  int64_t slab_floats = 0;  // padded floats per vP slab
  float *a = nullptr, *b = nullptr, *arrival = nullptr, *dense = nullptr;
  float *plane = nullptr, *last = nullptr;
  double *sn = nullptr, *cs = nullptr;
  float *snf = nullptr, *csf = nullptr;
  pe::Rel5Stats *stats = nullptr, *host_stats = nullptr;
  cudaStream_t own = nullptr, stream = nullptr;
  bool initialized = false;
};

namespace {

using pe::fail;

// Geometry of `slabs` consecutive vP slabs as a grid of their own (for the
// layout conversions and the initialisation, which do not look at vP).
pe::Rel5Grid view(const pe::Rel5Grid &g, int slabs) {
  pe::Rel5Grid v = g;
  v.nvp = slabs;
  v.n_padded = g.sv * slabs;
  v.n = (int64_t)g.nx * g.nx * g.nh * g.nve * slabs;
  return v;
}

void release(pe_relative_shard *h) {
  for (void *ptr : {(void *)h->a, (void *)h->b, (void *)h->arrival, (void *)h->dense,
                    (void *)h->plane, (void *)h->sn, (void *)h->cs, (void *)h->snf,
                    (void *)h->csf, (void *)h->stats})
    cudaFree(ptr);
  if (h->host_stats) cudaFreeHost(h->host_stats);
  if (h->own) cudaStreamDestroy(h->own);
}

int enter(pe_relative_shard *h) {
  if (!h) return fail(PE_EINVAL, "handle is NULL");
  PE_CUDA_TRY(cudaSetDevice(h->p.device));
  return PE_OK;
}

int read_stats(pe_relative_shard *h) {
  PE_CUDA_TRY(cudaMemcpyAsync(h->host_stats, h->stats, sizeof(pe::Rel5Stats),
                              cudaMemcpyDeviceToHost, h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (h->host_stats->timeout) return fail(PE_ETIMEOUT, "a bounded device wait gave up");
  if (h->host_stats->nonfinite) return fail(PE_ENONFINITE, "Nonfinite field update");
  return PE_OK;
}

// Owned slabs of a padded buffer -> host, dense.
int copy_owned(pe_relative_shard *h, const float *buffer, float *host) {
  const int n_own = h->own_hi - h->own_lo;
  const pe::Rel5Grid v = view(h->g, n_own);
  PE_CUDA_TRY(pe::rel5_pack(v, buffer + (h->own_lo - h->lo) * h->slab_floats, h->dense,
                            h->stream));
  pe::count_launches(1);
  PE_CUDA_TRY(cudaMemcpyAsync(host, h->dense, sizeof(float) * (size_t)v.n,
                              cudaMemcpyDeviceToHost, h->stream));
  return read_stats(h);
}

}  // namespace

extern "C" {

int pe_relative_shard_create(const pe_relative_params *params, int32_t vp_begin,
                             int32_t vp_end, pe_relative_shard **out) {
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = pe::rel5host::validate(params);
  if (rc) return rc;
  const int nvp = params->p_speeds, halo = params->order;
  if (vp_begin < 0 || vp_end > nvp || vp_begin >= vp_end)
    return fail(PE_EINVAL, "owned vP slabs must satisfy 0 <= begin < end <= p_speeds");
  if ((vp_begin > 0 || vp_end < nvp) && vp_end - vp_begin < halo)
    return fail(PE_EINVAL, "a shard with a neighbour must own at least `order` vP slabs");
  PE_CUDA_TRY(cudaSetDevice(params->device));
  pe_relative_shard *h = new pe_relative_shard();
  h->p = *params;
  h->g = pe::rel5host::make_grid(params);
  h->own_lo = vp_begin;
  h->own_hi = vp_end;
  h->lo = vp_begin - halo < 0 ? 0 : vp_begin - halo;
  h->hi = vp_end + halo > nvp ? nvp : vp_end + halo;
  h->g.own_lo = vp_begin;
  h->g.own_n = vp_end - vp_begin;
  h->g.slab_lo = h->lo;
  h->slab_floats = h->g.sv;
  h->tile = pe::rel5_default_tile(h->g);
  const int slabs = h->hi - h->lo, nh = h->g.nh;
  const size_t bytes = sizeof(float) * (size_t)h->g.sv * slabs;
  std::vector<double> sn(nh), cs(nh);
  std::vector<float> snf(nh), csf(nh);
  const double pi = std::acos(-1.0);
  for (int k = 0; k < nh; k++) {
    const double q = -pi + k * h->g.dphi;  // native_relative.cpp:84-89
    sn[k] = std::sin(q);
    cs[k] = std::cos(q);
    snf[k] = (float)sn[k];
    csf[k] = (float)cs[k];
  }
  cudaError_t err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  take(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
  h->stream = h->own;
  take(cudaMalloc(&h->a, bytes));
  take(cudaMalloc(&h->b, bytes));
  take(cudaMalloc(&h->arrival, bytes));
  take(cudaMalloc(&h->dense, bytes));
  take(cudaMalloc(&h->plane, sizeof(float) * (size_t)h->g.nx * h->g.nx));
  take(cudaMalloc(&h->sn, sizeof(double) * nh));
  take(cudaMalloc(&h->cs, sizeof(double) * nh));
  take(cudaMalloc(&h->snf, sizeof(float) * nh));
  take(cudaMalloc(&h->csf, sizeof(float) * nh));
  take(cudaMalloc(&h->stats, sizeof(pe::Rel5Stats)));
  take(cudaMallocHost(&h->host_stats, sizeof(pe::Rel5Stats)));
  if (err == cudaSuccess) {
    // halo slabs start at 0 until the first exchange fills them
    take(cudaMemset(h->a, 0, bytes));
    take(cudaMemset(h->b, 0, bytes));
    take(cudaMemcpy(h->sn, sn.data(), sizeof(double) * nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->cs, cs.data(), sizeof(double) * nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->snf, snf.data(), sizeof(float) * nh, cudaMemcpyHostToDevice));
    take(cudaMemcpy(h->csf, csf.data(), sizeof(float) * nh, cudaMemcpyHostToDevice));
    take(cudaMemset(h->stats, 0, sizeof(pe::Rel5Stats)));
  }
  if (err != cudaSuccess) {
    rc = pe::cuda_fail(err, "pe_relative_shard_create");
    release(h);
    delete h;
    return rc;
  }
  h->last = h->a;
  *out = h;
  return PE_OK;
}

int pe_relative_shard_layout(const pe_relative_shard *h, int32_t *slabs,
                             int64_t *slab_floats) {
  if (!h || !slabs) return fail(PE_EINVAL, "NULL argument");
  slabs[0] = h->lo;
  slabs[1] = h->hi;
  slabs[2] = h->own_lo;
  slabs[3] = h->own_hi;
  if (slab_floats) *slab_floats = h->slab_floats;
  return PE_OK;
}

int pe_relative_shard_set_stream(pe_relative_shard *h, void *cuda_stream) {
  int rc = enter(h);
  if (rc) return rc;
  h->stream = cuda_stream ? (cudaStream_t)cuda_stream : h->own;
  return PE_OK;
}

int pe_relative_shard_init(pe_relative_shard *h, const float *initial, double start_time) {
  int rc = enter(h);
  if (rc) return rc;
  if (!std::isfinite(start_time) || start_time < 0)
    return fail(PE_EINVAL, "start_time must be finite and >= 0");
  const pe::Rel5Grid v = view(h->g, h->hi - h->lo);
  PE_CUDA_TRY(cudaMemsetAsync(h->stats, 0, sizeof(pe::Rel5Stats), h->stream));
  if (!initial) {
    // the circular capture field (native_relative.cpp:91-100) on every slab
    const int nx = h->g.nx;
    std::vector<float> plane((size_t)nx * nx);
    for (int iy = 0; iy < nx; iy++) {
      const double y = -h->g.extent + iy * h->g.dx;
      for (int ix = 0; ix < nx; ix++)
        plane[(size_t)iy * nx + ix] =
            (float)(std::hypot(-h->g.extent + ix * h->g.dx, y) - h->p.capture_radius);
    }
    PE_CUDA_TRY(cudaMemcpyAsync(h->plane, plane.data(), sizeof(float) * plane.size(),
                                cudaMemcpyHostToDevice, h->stream));
    PE_CUDA_TRY(pe::rel5_init(v, h->plane, h->a, h->arrival, (float)start_time, h->stream));
    pe::count_launches(1);
  } else {
    PE_CUDA_TRY(cudaMemcpyAsync(h->dense, initial, sizeof(float) * (size_t)v.n,
                                cudaMemcpyHostToDevice, h->stream));
    PE_CUDA_TRY(pe::rel5_unpack(v, h->dense, h->a, h->stream));
    PE_CUDA_TRY(pe::rel5_init(v, nullptr, h->a, h->arrival, (float)start_time, h->stream));
    pe::count_launches(2);
  }
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->t = start_time;
  h->steps = 0;
  h->last = h->a;
  h->initialized = true;
  return PE_OK;
}

int pe_relative_shard_stage(pe_relative_shard *h, int32_t stage, double dt) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->initialized) return fail(PE_ESTATE, "stage before init");
  if (stage < 0 || stage >= h->g.order) return fail(PE_EINVAL, "stage must be in [0, order)");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(PE_EINVAL, "dt must be positive");
  if (stage == 0)
    PE_CUDA_TRY(cudaMemsetAsync(&h->stats->residual, 0, sizeof(unsigned long long),
                                h->stream));
  pe::Rel5Stage s{};
  const int blend = stage == 1;
  s.src = blend ? h->b : h->a;
  s.dst = blend ? h->a : h->b;
  s.arrival = h->arrival;
  s.sn = h->sn;
  s.cs = h->cs;
  s.snf = h->snf;
  s.csf = h->csf;
  s.dt = dt;
  s.t = h->t;
  s.stats = h->stats;
  PE_CUDA_TRY(h->p.precision == PE_LOCAL_F64
                  ? pe::rel5_stage_f64(h->g, s, blend, h->stream)
                  : pe::rel5_stage_f32(h->g, h->tile, s, blend, h->stream));
  pe::count_launches(1);
  h->last = s.dst;
  if (stage == h->g.order - 1) {
    if (h->g.order == 1) std::swap(h->a, h->b);  // the step's result is the field
    h->t += dt;
    h->steps += 1;
  }
  return PE_OK;
}

int pe_relative_shard_buffer(const pe_relative_shard *h, float **device_buffer) {
  if (!h || !device_buffer) return fail(PE_EINVAL, "NULL argument");
  *device_buffer = h->last;
  return PE_OK;
}

int pe_relative_shard_copy_field(pe_relative_shard *h, float *host_owned) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_owned) return fail(PE_EINVAL, "host buffer is NULL");
  return copy_owned(h, h->a, host_owned);
}

int pe_relative_shard_copy_arrival(pe_relative_shard *h, float *host_owned) {
  int rc = enter(h);
  if (rc) return rc;
  if (!host_owned) return fail(PE_EINVAL, "host buffer is NULL");
  return copy_owned(h, h->arrival, host_owned);
}

int pe_relative_shard_stats(pe_relative_shard *h, double *residual, double *increase) {
  int rc = enter(h);
  if (rc) return rc;
  rc = read_stats(h);
  if (rc) return rc;
  if (residual) std::memcpy(residual, &h->host_stats->residual, sizeof(double));
  if (increase) std::memcpy(increase, &h->host_stats->increase, sizeof(double));
  return PE_OK;
}

int pe_relative_shard_synchronize(pe_relative_shard *h) {
  int rc = enter(h);
  if (rc) return rc;
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_relative_shard_destroy(pe_relative_shard *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->p.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
