// Dense 8D ENO/Lax-Friedrichs stage on the GPU, float32 arithmetic in the
// order of native_world.cpp:32-74 (slopes) and :261-314 (stage).  This file
// is compiled with -fmad=false so that no multiply-add is fused: every stored
// float equals the reference CPU executable's bit for bit.
//
// The stage kernel itself is in world8d_stage.cuh (shared with the fast
// variant); this file holds its exact instantiation and the init kernels.
#include "world8d_stage.cuh"

namespace pe {
namespace {

// Separating-axis contact value of two oriented rectangles (double), in the
// order of the oracle's po_rect_separation.
__global__ void world8_contact_kernel(World8Grid g, const double *cs,
                                      const double *sn, const double *cdiff,
                                      const double *sdiff, double p_len,
                                      double p_wid, double e_len, double e_wid,
                                      double dxd, float *field,
                                      float *arrival) {
  const int64_t poses = g.cells / g.shape[7];  // speeds do not enter
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < poses;
       p += (int64_t)gridDim.x * blockDim.x) {
    // p enumerates [xP, yP, thP, vP, xE, yE, thE]
    int64_t rest = p;
    const int the = (int)(rest % g.shape[6]);
    rest /= g.shape[6];
    const int ye = (int)(rest % g.shape[5]);
    rest /= g.shape[5];
    const int xe = (int)(rest % g.shape[4]);
    rest /= g.shape[4];
    rest /= g.shape[3];  // vP
    const int thp = (int)(rest % g.shape[2]);
    rest /= g.shape[2];
    const int yp = (int)(rest % g.shape[1]);
    const int xp = (int)(rest / g.shape[1]);
    const double ext = (double)g.extent;
    const double px = -ext + xp * dxd, py = -ext + yp * dxd;
    const double ex = -ext + xe * dxd, ey = -ext + ye * dxd;
    const double d0 = ex - px, d1 = ey - py;
    // cos/sin of (thE - thP), tabulated on the host with the C library
    const double ca = fabs(cdiff[the * g.nh + thp]), sa = fabs(sdiff[the * g.nh + thp]);
    double best = -INFINITY;
    const int hk[2] = {thp, the};
    const double own_l[2] = {p_len, e_len}, own_w[2] = {p_wid, e_wid};
    const double oth_l[2] = {e_len, p_len}, oth_w[2] = {e_wid, p_wid};
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const double c = cs[hk[k]], s_ = sn[hk[k]];
      const double x = d0 * c + d1 * s_;
      const double y = -d0 * s_ + d1 * c;
      const double gx = fabs(x) - own_l[k] / 2 - (oth_l[k] * ca + oth_w[k] * sa) / 2;
      const double gy = fabs(y) - own_w[k] / 2 - (oth_l[k] * sa + oth_w[k] * ca) / 2;
      if (gx > best) best = gx;
      if (gy > best) best = gy;
    }
    const float value = (float)best;
    for (int v = 0; v < g.shape[7]; v++) {
      field[p * g.shape[7] + v] = value;
      arrival[p * g.shape[7] + v] = value <= 0 ? 0.f : __int_as_float(0x7fc00000);
    }
  }
}

__global__ void world8_square_kernel(World8Grid g, const float *x, float radius,
                                     float *field, float *arrival) {
  const int64_t block = (int64_t)g.shape[6] * g.shape[7];
  const int64_t blocks = g.cells / block;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < blocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    int64_t rest = b;
    const int ye = (int)(rest % g.shape[5]);
    rest /= g.shape[5];
    const int xe = (int)(rest % g.shape[4]);
    rest /= g.shape[4];
    rest /= g.shape[3];
    rest /= g.shape[2];
    const int yp = (int)(rest % g.shape[1]);
    const int xp = (int)(rest / g.shape[1]);
    const float capture = hypotf(x[xp] - x[xe], x[yp] - x[ye]) - radius;
    const float axe = fabsf(x[xe]), aye = fabsf(x[ye]);
    const float e_fault = g.arena - (axe < aye ? aye : axe);
    const float target = e_fault < capture ? e_fault : capture;
    const float axp = fabsf(x[xp]), ayp = fabsf(x[yp]);
    const float avoid = (axp < ayp ? ayp : axp) - g.arena + 1e-6f;
    const float initial = target < avoid ? avoid : target;
    for (int64_t k = 0; k < block; k++) {
      field[b * block + k] = initial;
      arrival[b * block + k] = initial <= 0 ? 0.f : __int_as_float(0x7fc00000);
    }
  }
}

__global__ void world8_arrival_kernel(int64_t n, const float *field,
                                      float *arrival, float start) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    arrival[j] = field[j] <= 0 ? start : __int_as_float(0x7fc00000);
}

}  // namespace

cudaError_t world8_stage(const World8Grid &g, const World8Stage &s,
                         cudaStream_t stream) {
  return w8::launch_stage<false>(g, s, stream);
}

cudaError_t world8_init_contact(const World8Grid &g, const double *cs,
                                const double *sn, const double *cdiff,
                                const double *sdiff, double p_len, double p_wid,
                                double e_len, double e_wid, float *field,
                                float *arrival, cudaStream_t stream) {
  const double dxd = 2 * (double)g.extent / (g.n - 1);
  world8_contact_kernel<<<148 * 8, 256, 0, stream>>>(g, cs, sn, cdiff, sdiff, p_len,
                                                     p_wid, e_len, e_wid, dxd, field,
                                                     arrival);
  return cudaGetLastError();
}

cudaError_t world8_init_square(const World8Grid &g, const float *x,
                               float radius, float *field, float *arrival,
                               cudaStream_t stream) {
  world8_square_kernel<<<148 * 8, 256, 0, stream>>>(g, x, radius, field, arrival);
  return cudaGetLastError();
}

namespace {

__global__ void world8_map_kernel(const World8Grid g, float radius,
                                  const float *__restrict__ p_clear,
                                  const float *__restrict__ e_clear, float *__restrict__ field,
                                  float *__restrict__ arrival) {
  const float dx = 2 * g.extent / (g.n - 1);
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < g.cells;
       j += (int64_t)gridDim.x * blockDim.x) {
    int q[8];
    int64_t rest = j;
    for (int k = 7; k >= 0; k--) {
      q[k] = (int)(rest % g.shape[k]);
      rest /= g.shape[k];
    }
    const float cap = hypotf((q[0] - q[4]) * dx, (q[1] - q[5]) * dx) - radius;
    const float p = p_clear[(q[0] * g.n + q[1]) * g.nh + q[2]];
    const float e = e_clear[(q[4] * g.n + q[5]) * g.nh + q[6]];
    const float v = fmaxf(fminf(cap, e), -p + 1e-6f);
    field[j] = v;
    arrival[j] = v <= 0 ? 0.f : __int_as_float(0x7fc00000);
  }
}

}  // namespace

cudaError_t world8_init_map(const World8Grid &g, float radius, const float *p_clear,
                            const float *e_clear, float *field, float *arrival,
                            cudaStream_t stream) {
  world8_map_kernel<<<148 * 8, 256, 0, stream>>>(g, radius, p_clear, e_clear, field, arrival);
  return cudaGetLastError();
}

cudaError_t world8_init_arrival(const World8Grid &g, const float *field,
                                float *arrival, float start,
                                cudaStream_t stream) {
  world8_arrival_kernel<<<148 * 8, 256, 0, stream>>>(g.cells, field, arrival, start);
  return cudaGetLastError();
}

}  // namespace pe
