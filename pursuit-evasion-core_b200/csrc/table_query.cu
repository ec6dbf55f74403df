// Queries of a completed relative table on the GPU (pe_table_*): the signed
// field at a budget and the capture time of arbitrary relative states,
// with the semantics of the reference reader
// (reversible/relative_table.py:76-161), the table resident in HBM.
//
// Per state: a 32-corner multilinear stencil over [vP, vE, psi, y, x]
// (periodic heading, speeds and positions clamped to the box, weights
// multiplied in axis order), in double; capture time = first zero
// crossing by bisection over the frames, then linear interpolation between
// the bracketing frames.  The reference bisects the whole batch at once,
// so a state whose bracket has closed keeps taking "mid = lo" steps while
// any other state of the batch still bisects; the result differs only for
// a state whose earliest frame is already inside.  The GPU path reproduces
// that: pass 1 bisects every state on its own and records its step count,
// pass 2 applies the extra steps implied by the batch's maximum.
#include <cmath>
#include <vector>

#include "pe_internal.h"

struct pe_table {
  int device = 0;
  int frames = 0;
  int64_t cells = 0;
  float *fields = nullptr;  // [frames][cells]
  double *times = nullptr;  // [frames]
  int shape[5];
  double lo[5], hi[5], h[5];  // per storage axis [vP, vE, psi, y, x]
  double radius = 0, p_min = 0, p_max = 0, e_min = 0, e_max = 0;
  // per-query scratch, grown on demand
  double *states = nullptr, *out = nullptr, *budget = nullptr, *ab = nullptr;
  int *bracket = nullptr, *flags = nullptr, *max_steps = nullptr;
  int64_t capacity = 0;
  cudaStream_t stream = nullptr;
};

namespace pe {
namespace {

struct TableView {
  const float *fields;
  const double *times;
  int64_t cells;
  int frames;
  int shape[5];
  int64_t stride[5];
  double lo[5], hi[5], h[5];
  double radius, p_min, p_max, e_min, e_max;
};

// Stencil of one state (x, y, psi, vP, vE): flat corner indices and
// weights; false if the state is not finite or outside the box.
__device__ bool stencil(const TableView &t, const double *s, int64_t idx[32], double w[32]) {
  const double q[5] = {s[3], s[4], s[2], s[1], s[0]};  // storage order
  bool valid = true;
  double frac[5];
  int lower[5];
  for (int k = 0; k < 5; k++) {
    valid &= isfinite(q[k]);
    const double v = isfinite(q[k]) ? q[k] : 0.0;
    if (k == 2) {
      const double twopi = 2 * M_PI;
      double r = fmod(v + M_PI, twopi);
      if (r < 0) r += twopi;  // Python's modulo takes the divisor's sign
      const double f = r / t.h[k];
      const double fl = floor(f);
      int l = (int)fmod(fl, (double)t.shape[k]);
      if (l < 0) l += t.shape[k];
      lower[k] = l;
      frac[k] = f - fl;
    } else {
      valid &= v >= t.lo[k] - 1e-10 && v <= t.hi[k] + 1e-10;
      const double c = fmin(fmax(v, t.lo[k]), t.hi[k]);
      const double f = (c - t.lo[k]) / t.h[k];
      const int l = min((int)floor(f), t.shape[k] - 2);
      lower[k] = l;
      frac[k] = f - l;
    }
  }
  for (int c = 0; c < 32; c++) {
    int64_t i = 0;
    double wt = 1.0;
    for (int k = 0; k < 5; k++) {
      const int bit = (c >> (4 - k)) & 1;  // corner bits in axis order, last fastest
      int corner = lower[k] + bit;
      if (k == 2) corner %= t.shape[k];
      i += (int64_t)corner * t.stride[k];
      wt *= bit ? frac[k] : 1.0 - frac[k];
    }
    idx[c] = i;
    w[c] = wt;
  }
  return valid;
}

__device__ double sample(const TableView &t, int frame, const int64_t idx[32],
                         const double w[32]) {
  const float *f = t.fields + (int64_t)frame * t.cells;
  double sum = 0;
  for (int c = 0; c < 32; c++) sum += (double)f[idx[c]] * w[c];
  return sum;
}

__device__ bool physical(const TableView &t, const double *s) {
  bool ok = true;
  for (int k = 0; k < 5; k++) ok &= isfinite(s[k]);
  ok &= s[3] >= t.p_min - 1e-10 && s[3] <= t.p_max + 1e-10;
  ok &= s[4] >= t.e_min - 1e-10 && s[4] <= t.e_max + 1e-10;
  return ok;
}

// flags: bit 0 stencil valid, bit 1 still valid after the horizon test,
// bit 2 captured and physical, bits 3.. this state's bisection steps.
__global__ void value_pass1(TableView t, const double *states, int64_t n, int *bracket,
                            double *ab, int *flags, int *max_steps) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *s = states + 5 * i;
  int64_t idx[32];
  double w[32];
  const bool valid = stencil(t, s, idx, w);
  int lo = 0, hi = t.frames - 1, steps = 0;
  const bool inside_end = sample(t, hi, idx, w) <= 0;
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (sample(t, mid, idx, w) <= 0)
      hi = mid;
    else
      lo = mid;
    steps++;
  }
  bracket[2 * i] = lo;
  bracket[2 * i + 1] = hi;
  ab[2 * i] = sample(t, lo, idx, w);
  ab[2 * i + 1] = sample(t, hi, idx, w);
  const double r = sqrt(__dadd_rn(__dmul_rn(s[0], s[0]), __dmul_rn(s[1], s[1])));
  const bool captured = r <= t.radius && physical(t, s);
  flags[i] = (valid ? 1 : 0) | (valid && inside_end ? 2 : 0) | (captured ? 4 : 0) |
             (steps << 3);
  atomicMax(max_steps, steps);
}

__global__ void value_pass2(TableView t, int64_t n, const int *bracket, const double *ab,
                            const int *flags, const int *max_steps, int any_valid,
                            double *out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = flags[i];
  if (!any_valid) {
    out[i] = (f & 4) ? 0.0 : NAN;
    return;
  }
  int lo = bracket[2 * i], hi = bracket[2 * i + 1];
  double a = ab[2 * i], b = ab[2 * i + 1];
  // the batch kept bisecting: with a closed bracket mid = lo, and an
  // inside lo pulls hi down to it
  if ((f >> 3) < *max_steps && hi - lo == 1 && a <= 0) {
    hi = lo;
    b = a;
  }
  const double frac = fabs(a - b) > 1e-14 ? a / (a - b) : 0.0;
  double v = t.times[lo] + fmin(fmax(frac, 0.0), 1.0) * (t.times[hi] - t.times[lo]);
  if (!(f & 2)) v = NAN;
  out[i] = (f & 4) ? 0.0 : v;
}

__global__ void field_kernel(TableView t, const double *states, const double *budget,
                             int64_t n, double *out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t idx[32];
  double w[32];
  bool valid = stencil(t, states + 5 * i, idx, w);
  double tau = budget[i];
  const double horizon = t.times[t.frames - 1];
  valid &= isfinite(tau) && tau >= 0 && tau <= horizon + 1e-10;
  if (!isfinite(tau)) tau = 0;
  // searchsorted(times, tau, side="right") - 1, clipped to [0, frames - 2]
  int k = 0;
  while (k + 1 < t.frames && t.times[k + 1] <= tau) k++;
  k = max(0, min(k, t.frames - 2));
  const double frac = (tau - t.times[k]) / (t.times[k + 1] - t.times[k]);
  const double a = sample(t, k, idx, w), b = sample(t, k + 1, idx, w);
  out[i] = valid ? a + frac * (b - a) : NAN;
}

TableView view(const pe_table *h) {
  TableView t{};
  t.fields = h->fields;
  t.times = h->times;
  t.cells = h->cells;
  t.frames = h->frames;
  int64_t stride = 1;
  for (int k = 4; k >= 0; k--) {
    t.shape[k] = h->shape[k];
    t.stride[k] = stride;
    stride *= h->shape[k];
    t.lo[k] = h->lo[k];
    t.hi[k] = h->hi[k];
    t.h[k] = h->h[k];
  }
  t.radius = h->radius;
  t.p_min = h->p_min;
  t.p_max = h->p_max;
  t.e_min = h->e_min;
  t.e_max = h->e_max;
  return t;
}

int reserve(pe_table *h, int64_t n) {
  if (n <= h->capacity) return PE_OK;
  for (void *p : {(void *)h->states, (void *)h->out, (void *)h->budget, (void *)h->ab,
                  (void *)h->bracket, (void *)h->flags})
    cudaFree(p);
  h->states = h->out = h->budget = h->ab = nullptr;
  h->bracket = h->flags = nullptr;
  h->capacity = 0;
  PE_CUDA_TRY(cudaMalloc(&h->states, sizeof(double) * 5 * n));
  PE_CUDA_TRY(cudaMalloc(&h->out, sizeof(double) * n));
  PE_CUDA_TRY(cudaMalloc(&h->budget, sizeof(double) * n));
  PE_CUDA_TRY(cudaMalloc(&h->ab, sizeof(double) * 2 * n));
  PE_CUDA_TRY(cudaMalloc(&h->bracket, sizeof(int) * 2 * n));
  PE_CUDA_TRY(cudaMalloc(&h->flags, sizeof(int) * n));
  h->capacity = n;
  return PE_OK;
}

void release(pe_table *h) {
  for (void *p : {(void *)h->fields, (void *)h->times, (void *)h->states, (void *)h->out,
                  (void *)h->budget, (void *)h->ab, (void *)h->bracket, (void *)h->flags,
                  (void *)h->max_steps})
    cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace
}  // namespace pe

extern "C" {

int pe_table_create(const float *host_frames, int32_t frames, const double *times,
                    const int32_t shape[5], const double axis_lo[5], const double axis_hi[5],
                    const double spacing[5], double capture_radius,
                    const double speed_limits[4], int32_t device, pe_table **out) {
  using pe::fail;
  if (!out) return fail(PE_EINVAL, "out is NULL");
  *out = nullptr;
  if (!host_frames || !times || !shape || !axis_lo || !axis_hi || !spacing || !speed_limits ||
      frames < 2)
    return fail(PE_EINVAL, "table: frames >= 2 and every array required");
  int64_t cells = 1;
  for (int k = 0; k < 5; k++) {
    if (shape[k] < 2 || !(spacing[k] > 0)) return fail(PE_EINVAL, "table: invalid axis %d", k);
    cells *= shape[k];
  }
  for (int f = 1; f < frames; f++)
    if (!(times[f] > times[f - 1])) return fail(PE_EINVAL, "table: times must increase");
  PE_CUDA_TRY(cudaSetDevice(device));
  pe_table *h = new pe_table();
  h->device = device;
  h->frames = frames;
  h->cells = cells;
  for (int k = 0; k < 5; k++) {
    h->shape[k] = shape[k];
    h->lo[k] = axis_lo[k];
    h->hi[k] = axis_hi[k];
    h->h[k] = spacing[k];
  }
  h->radius = capture_radius;
  h->p_min = speed_limits[0];
  h->p_max = speed_limits[1];
  h->e_min = speed_limits[2];
  h->e_max = speed_limits[3];
  cudaError_t err = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaMalloc(&h->fields, sizeof(float) * (size_t)cells * frames);
  if (err == cudaSuccess) err = cudaMalloc(&h->times, sizeof(double) * frames);
  if (err == cudaSuccess) err = cudaMalloc(&h->max_steps, sizeof(int));
  if (err == cudaSuccess)
    err = cudaMemcpy(h->fields, host_frames, sizeof(float) * (size_t)cells * frames,
                     cudaMemcpyHostToDevice);
  if (err == cudaSuccess)
    err = cudaMemcpy(h->times, times, sizeof(double) * frames, cudaMemcpyHostToDevice);
  if (err != cudaSuccess) {
    const int rc = pe::cuda_fail(err, "pe_table_create");
    pe::release(h);
    delete h;
    return rc;
  }
  *out = h;
  return PE_OK;
}

int pe_table_value(pe_table *h, const double *host_states, int64_t n, double *host_out) {
  using pe::fail;
  if (!h || !host_states || !host_out || n <= 0) return fail(PE_EINVAL, "table: invalid query");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  int rc = pe::reserve(h, n);
  if (rc) return rc;
  PE_CUDA_TRY(cudaMemcpyAsync(h->states, host_states, sizeof(double) * 5 * n,
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaMemsetAsync(h->max_steps, 0, sizeof(int), h->stream));
  const pe::TableView t = pe::view(h);
  const int threads = 128;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  pe::value_pass1<<<blocks, threads, 0, h->stream>>>(t, h->states, n, h->bracket, h->ab,
                                                      h->flags, h->max_steps);
  PE_CUDA_TRY(cudaGetLastError());
  // any stencil-valid state? (the reference returns early otherwise)
  std::vector<int> flags(n);
  PE_CUDA_TRY(cudaMemcpyAsync(flags.data(), h->flags, sizeof(int) * n, cudaMemcpyDeviceToHost,
                              h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  int any = 0;
  for (int64_t i = 0; i < n && !any; i++) any = flags[i] & 1;
  pe::value_pass2<<<blocks, threads, 0, h->stream>>>(t, n, h->bracket, h->ab, h->flags,
                                                      h->max_steps, any, h->out);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(2);
  PE_CUDA_TRY(cudaMemcpyAsync(host_out, h->out, sizeof(double) * n, cudaMemcpyDeviceToHost,
                              h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_table_field(pe_table *h, const double *host_states, const double *host_budgets,
                   int64_t n, double *host_out) {
  using pe::fail;
  if (!h || !host_states || !host_budgets || !host_out || n <= 0)
    return fail(PE_EINVAL, "table: invalid query");
  PE_CUDA_TRY(cudaSetDevice(h->device));
  int rc = pe::reserve(h, n);
  if (rc) return rc;
  PE_CUDA_TRY(cudaMemcpyAsync(h->states, host_states, sizeof(double) * 5 * n,
                              cudaMemcpyHostToDevice, h->stream));
  PE_CUDA_TRY(cudaMemcpyAsync(h->budget, host_budgets, sizeof(double) * n,
                              cudaMemcpyHostToDevice, h->stream));
  const int threads = 128;
  pe::field_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, h->stream>>>(
      pe::view(h), h->states, h->budget, n, h->out);
  PE_CUDA_TRY(cudaGetLastError());
  pe::count_launches(1);
  PE_CUDA_TRY(cudaMemcpyAsync(host_out, h->out, sizeof(double) * n, cudaMemcpyDeviceToHost,
                              h->stream));
  PE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return PE_OK;
}

int pe_table_destroy(pe_table *h) {
  if (!h) return PE_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  pe::release(h);
  delete h;
  return PE_OK;
}

}  // extern "C"
