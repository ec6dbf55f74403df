// Vehicle geometry of the compact contact game on the GPU: obstacle
// clearance of a rectangular car in a square arena with circular obstacles,
// held-command arcs, swept-motion safety, braking backups and straight
// configuration-space connections.  The grid construction of the compact
// game (make_grid, local_game/grid_game.py:158-196) asks these for every
// (state, control) of a vehicle grid -- tens of thousands of states times 9
// controls, each a recursive interval search -- so they run one thread per
// query here.
//
// Semantics (the game's definition, local_game/native_geometry.cpp:8-117,
// :221-246, and reversible/model.py:86-153 for the arc):
//   arc          acceleration held until the speed limit, then constant
//                speed; turn = curvature * signed distance; chord through
//                the mid heading; heading wrapped to [-pi, pi];
//   clearance    min of the two wall gaps of the rotated rectangle's
//                half extents and, per circle near enough to matter, the
//                signed rectangle/circle distance;
//   motion safe  the clearance along the arc over [0, t] stays positive:
//                an interval is safe when both end clearances exceed half
//                its length times a Lipschitz bound of the clearance
//                (speed times (1 + half diagonal * |curvature|)), unsafe
//                when an end clearance is <= 1e-7, and split otherwise, to
//                depth 18 or a length of 1e-8 (then unsafe);
//   backup safe  clear now and, unless stopped, one of three braking arcs
//                (straight, or either full curvature) to rest within the
//                control periods of maximal braking is motion safe;
//   connection   the straight interpolation between two configurations
//                (heading by the wrapped difference) stays clear, by the
//                same interval rule to depth 20.
// The interval searches are iterative with an explicit stack (the result
// is the conjunction of all leaves, so the visiting order does not matter).
// Double arithmetic without contraction (this file is built with
// -fmad=false), so decisions match the CPU formulation except where a
// clearance sits within rounding of a threshold.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pe_internal.h"

namespace {

struct Model {
  double v_lo, v_hi, acc, curv, length, width, dt;
};

constexpr double kTwoPi = 6.283185307179586476925286766559;

__device__ void arc(const double *s, double a, double k, double t, const Model &m,
                    double *out) {
  const double limit = a >= 0 ? m.v_hi : m.v_lo;
  const double hit = fabs(a) > 1e-14 ? (limit - s[3]) / a : INFINITY;
  const double held = fmin(t, fmax(0.0, hit));
  const double v = fmax(m.v_lo, fmin(m.v_hi, s[3] + a * t));
  const double dist = s[3] * held + 0.5 * a * held * held + v * (t - held);
  const double turn = k * dist;
  const double half = 0.5 * turn;
  const double chord = fabs(half) > 1e-12 ? sin(half) / half : 1.0;
  out[0] = s[0] + dist * chord * cos(s[2] + half);
  out[1] = s[1] + dist * chord * sin(s[2] + half);
  out[2] = remainder(s[2] + turn, kTwoPi);
  out[3] = v;
}

__device__ double clearance(const double *s, const double *circles, int nc, double half_width,
                            const Model &m) {
  const double c = cos(s[2]), q = sin(s[2]);
  const double hx = 0.5 * (m.length * fabs(c) + m.width * fabs(q));
  const double hy = 0.5 * (m.length * fabs(q) + m.width * fabs(c));
  double best = fmin(half_width - fabs(s[0]) - hx, half_width - fabs(s[1]) - hy);
  const double reach = 0.5 * hypot(m.length, m.width);
  for (int j = 0; j < nc; j++) {
    const double dx = circles[3 * j] - s[0], dy = circles[3 * j + 1] - s[1];
    const double r = circles[3 * j + 2];
    const double near = reach + r + fmax(0.0, best);
    if (dx * dx + dy * dy > near * near) continue;  // cannot lower the minimum
    const double along = fabs(dx * c + dy * q) - 0.5 * m.length;
    const double across = fabs(-dx * q + dy * c) - 0.5 * m.width;
    const double gap = hypot(fmax(0.0, along), fmax(0.0, across)) +
                       fmin(fmax(along, across), 0.0) - r;
    best = fmin(best, gap);
  }
  return best;
}

struct Span {
  double lo, hi, c_lo, c_hi;
  int depth;
};

// Clearance along the arc of (a, k) from s over [0, t] stays positive.
__device__ bool sweep_safe(const double *s, double a, double k, double t, const double *circles,
                           int nc, double half_width, const Model &m) {
  double end[4];
  arc(s, a, k, t, m, end);
  const double lip = fmax(fabs(s[3]), fabs(end[3])) *
                     (1.0 + 0.5 * hypot(m.length, m.width) * fabs(k));
  Span stack[24];
  int top = 0;
  stack[top++] = {0.0, t, clearance(s, circles, nc, half_width, m),
                  clearance(end, circles, nc, half_width, m), 0};
  while (top > 0) {
    const Span sp = stack[--top];
    const double low = fmin(sp.c_lo, sp.c_hi);
    if (low <= 1e-7) return false;
    if (low > lip * (sp.hi - sp.lo) * 0.5 + 1e-7) continue;
    if (sp.depth >= 18 || sp.hi - sp.lo < 1e-8) return false;
    const double mid = 0.5 * (sp.lo + sp.hi);
    double z[4];
    arc(s, a, k, mid, m, z);
    const double cm = clearance(z, circles, nc, half_width, m);
    stack[top++] = {mid, sp.hi, cm, sp.c_hi, sp.depth + 1};
    stack[top++] = {sp.lo, mid, sp.c_lo, cm, sp.depth + 1};
  }
  return true;
}

__device__ bool backup_safe(const double *s, const double *circles, int nc, double half_width,
                            const Model &m) {
  if (clearance(s, circles, nc, half_width, m) <= 1e-7) return false;
  if (fabs(s[3]) < 1e-10) return true;
  // braking at the full rate, held per control period, the last period's
  // command stopping exactly at its end; the arc depends only on the
  // distance, so one constant deceleration over the same distance traces it
  const double speed = fabs(s[3]);
  const int periods = max(1, (int)ceil(speed / (m.acc * m.dt) - 1e-10));
  const double full = (periods - 1) * m.dt, last = speed - m.acc * full;
  const double dist = speed * full - 0.5 * m.acc * full * full + 0.5 * last * m.dt;
  const double t = 2.0 * dist / speed, a = -s[3] / t;
  const double curvatures[3] = {0.0, -m.curv, m.curv};
  for (int q = 0; q < 3; q++)
    if (sweep_safe(s, a, curvatures[q], t, circles, nc, half_width, m)) return true;
  return false;
}

__device__ double lerp_clearance(const double *a, const double *b, double u, double angle,
                                 const double *circles, int nc, double half_width,
                                 const Model &m) {
  const double s[4] = {a[0] + u * (b[0] - a[0]), a[1] + u * (b[1] - a[1]), a[2] + u * angle,
                       0.0};
  return clearance(s, circles, nc, half_width, m);
}

__device__ bool connected(const double *a, const double *b, const double *circles, int nc,
                          double half_width, const Model &m) {
  const double angle = remainder(b[2] - a[2], kTwoPi);
  const double lip = hypot(b[0] - a[0], b[1] - a[1]) +
                     0.5 * hypot(m.length, m.width) * fabs(angle);
  Span stack[24];
  int top = 0;
  stack[top++] = {0.0, 1.0, clearance(a, circles, nc, half_width, m),
                  clearance(b, circles, nc, half_width, m), 0};
  while (top > 0) {
    const Span sp = stack[--top];
    const double low = fmin(sp.c_lo, sp.c_hi);
    if (low <= 1e-7) return false;
    if (low > lip * (sp.hi - sp.lo) * 0.5 + 1e-7) continue;
    if (sp.depth >= 20) return false;
    const double mid = 0.5 * (sp.lo + sp.hi);
    const double cm = lerp_clearance(a, b, mid, angle, circles, nc, half_width, m);
    stack[top++] = {mid, sp.hi, cm, sp.c_hi, sp.depth + 1};
    stack[top++] = {sp.lo, mid, sp.c_lo, cm, sp.depth + 1};
  }
  return true;
}

enum Query { kClearance = 0, kBackup = 1, kActions = 2, kConnections = 3 };

struct Args {
  Model m;
  const double *states, *targets, *controls, *circles;
  int64_t n;
  int na, nc;
  double half_width, dt;
  double *values, *next;
  uint8_t *flags;
};

template <int Q>
__global__ void __launch_bounds__(128) geometry_kernel(const Args g) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t count = Q == kActions ? g.n * g.na : g.n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += stride) {
    if (Q == kClearance) {
      g.values[i] = clearance(g.states + 4 * i, g.circles, g.nc, g.half_width, g.m);
    } else if (Q == kBackup) {
      g.flags[i] = backup_safe(g.states + 4 * i, g.circles, g.nc, g.half_width, g.m);
    } else if (Q == kActions) {
      const int64_t st = i / g.na;
      const int u = (int)(i - st * g.na);
      const double *s = g.states + 4 * st;
      const double a = g.controls[2 * u], k = g.controls[2 * u + 1];
      double *out = g.next + 4 * i;
      arc(s, a, k, g.dt, g.m, out);
      g.flags[i] = sweep_safe(s, a, k, g.dt, g.circles, g.nc, g.half_width, g.m) &&
                   backup_safe(out, g.circles, g.nc, g.half_width, g.m);
    } else {
      g.flags[i] = connected(g.states + 4 * i, g.targets + 4 * i, g.circles, g.nc,
                             g.half_width, g.m);
    }
  }
}

// Device copies of the inputs, one launch, results back to the host.
template <int Q>
int run(const pe_vehicle_model *model, const double *states, const double *targets,
        int64_t n, const double *controls, int32_t na, double dt, const double *circles,
        int32_t nc, double half_width, double *values, uint8_t *flags, double *next,
        int32_t device, const char *what) {
  using pe::fail;
  if (!model || !states || n < 0 || nc < 0 || (nc > 0 && !circles))
    return fail(PE_EINVAL, "%s: invalid arguments", what);
  if (!(half_width > 0) || !std::isfinite(half_width))
    return fail(PE_EINVAL, "%s: half_width must be positive", what);
  if (n == 0) return PE_OK;
  const int64_t outs = Q == kActions ? n * (int64_t)na : n;
  if (Q == kActions && (na <= 0 || !controls || !next || !(dt > 0)))
    return fail(PE_EINVAL, "%s: controls, next and dt > 0 are required", what);
  if (Q == kConnections && !targets) return fail(PE_EINVAL, "%s: targets required", what);
  if ((Q == kClearance && !values) || (Q != kClearance && !flags))
    return fail(PE_EINVAL, "%s: output buffer required", what);
  PE_CUDA_TRY(cudaSetDevice(device));
  Args g{};
  g.m = {model->speed_min, model->speed_max, model->acceleration, model->max_curvature,
         model->length, model->width, model->control_dt};
  g.n = n;
  g.na = na;
  g.nc = nc;
  g.half_width = half_width;
  g.dt = dt;
  std::vector<void *> owned;
  cudaError_t err = cudaSuccess;
  auto upload = [&](const double *src, size_t count) -> const double * {
    if (!src || count == 0 || err != cudaSuccess) return nullptr;
    void *p = nullptr;
    err = cudaMalloc(&p, sizeof(double) * count);
    if (err == cudaSuccess) {
      owned.push_back(p);
      err = cudaMemcpy(p, src, sizeof(double) * count, cudaMemcpyHostToDevice);
    }
    return static_cast<const double *>(p);
  };
  auto scratch = [&](size_t bytes) -> void * {
    if (err != cudaSuccess) return nullptr;
    void *p = nullptr;
    err = cudaMalloc(&p, bytes);
    if (err == cudaSuccess) owned.push_back(p);
    return p;
  };
  g.states = upload(states, 4 * (size_t)n);
  g.targets = Q == kConnections ? upload(targets, 4 * (size_t)n) : nullptr;
  g.controls = Q == kActions ? upload(controls, 2 * (size_t)na) : nullptr;
  g.circles = upload(circles, 3 * (size_t)nc);
  if (Q == kClearance) g.values = static_cast<double *>(scratch(sizeof(double) * outs));
  else g.flags = static_cast<uint8_t *>(scratch((size_t)outs));
  if (Q == kActions) g.next = static_cast<double *>(scratch(sizeof(double) * 4 * outs));
  if (err == cudaSuccess) {
    const int64_t blocks = std::min<int64_t>((outs + 127) / 128, 148 * 64);
    geometry_kernel<Q><<<(unsigned)blocks, 128>>>(g);
    pe::count_launches(1);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaDeviceSynchronize();
  if (err == cudaSuccess && Q == kClearance)
    err = cudaMemcpy(values, g.values, sizeof(double) * outs, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess && Q != kClearance)
    err = cudaMemcpy(flags, g.flags, (size_t)outs, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess && Q == kActions)
    err = cudaMemcpy(next, g.next, sizeof(double) * 4 * outs, cudaMemcpyDeviceToHost);
  for (void *p : owned) cudaFree(p);
  if (err != cudaSuccess) return pe::cuda_fail(err, what);
  return PE_OK;
}

}  // namespace

extern "C" {

int pe_geometry_clearance(const pe_vehicle_model *model, const double *states, int64_t n,
                          const double *circles, int32_t n_circles, double half_width,
                          double *out, int32_t device) {
  return run<kClearance>(model, states, nullptr, n, nullptr, 0, 0, circles, n_circles,
                         half_width, out, nullptr, nullptr, device, "pe_geometry_clearance");
}

int pe_geometry_backup_safe(const pe_vehicle_model *model, const double *states, int64_t n,
                            const double *circles, int32_t n_circles, double half_width,
                            uint8_t *out, int32_t device) {
  return run<kBackup>(model, states, nullptr, n, nullptr, 0, 0, circles, n_circles,
                      half_width, nullptr, out, nullptr, device, "pe_geometry_backup_safe");
}

int pe_geometry_actions(const pe_vehicle_model *model, const double *states, int64_t n,
                        const double *controls, int32_t n_controls, double dt,
                        const double *circles, int32_t n_circles, double half_width,
                        uint8_t *ok, double *next, int32_t device) {
  return run<kActions>(model, states, nullptr, n, controls, n_controls, dt, circles,
                       n_circles, half_width, nullptr, ok, next, device,
                       "pe_geometry_actions");
}

int pe_geometry_connections(const pe_vehicle_model *model, const double *from,
                            const double *to, int64_t n, const double *circles,
                            int32_t n_circles, double half_width, uint8_t *out,
                            int32_t device) {
  return run<kConnections>(model, from, to, n, nullptr, 0, 0, circles, n_circles, half_width,
                           nullptr, out, nullptr, device, "pe_geometry_connections");
}

}  // extern "C"
