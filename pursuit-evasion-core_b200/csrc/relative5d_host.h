// Host-side helpers of the relative 5D solvers shared by the single-grid
// handle (capi_relative.cu) and the batched handle (capi_batch.cu): option
// validation (native_relative.cpp:263-268), the padded device grid, the CFL
// step limit (native_relative.cpp:70-81) and the heading / capture tables
// (native_relative.cpp:84-100).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <initializer_list>
#include <vector>

#include "pe_internal.h"
#include "relative5d.cuh"

namespace pe {
namespace rel5host {

inline bool finite_all(std::initializer_list<double> values) {
  for (double v : values)
    if (!std::isfinite(v)) return false;
  return true;
}

inline int validate(const pe_relative_params *p) {
  if (!p) return pe::fail(PE_EINVAL, "params is NULL");
  if (p->positions < 3 || p->headings < 4 || p->p_speeds < 3 ||
      p->e_speeds < 3)
    return pe::fail(PE_EINVAL,
                "Invalid solver options: grid needs positions>=3, headings>=4, "
                "speeds>=3");
  if (p->order != 1 && p->order != 2)
    return pe::fail(PE_EINVAL, "Invalid solver options: order must be 1 or 2");
  if (p->scheme != PE_SCHEME_ENO_LF)
    return pe::fail(PE_EINVAL, "Invalid solver options: unknown scheme %d",
                p->scheme);
  if (p->precision != PE_LOCAL_F32 && p->precision != PE_LOCAL_F64)
    return pe::fail(PE_EINVAL, "Invalid solver options: unknown precision %d",
                p->precision);
  if (!finite_all({p->extent, p->capture_radius, p->p_speed_min,
                   p->p_speed_max, p->p_acceleration, p->p_curvature,
                   p->e_speed_min, p->e_speed_max, p->e_acceleration,
                   p->e_curvature, p->cfl}))
    return pe::fail(PE_EINVAL, "Invalid solver options: non-finite value");
  if (p->extent <= p->capture_radius || p->capture_radius <= 0 ||
      p->cfl <= 0 || p->cfl > 1 || p->p_acceleration <= 0 ||
      p->e_acceleration <= 0 || p->p_curvature <= 0 || p->e_curvature <= 0 ||
      p->p_speed_min >= p->p_speed_max || p->e_speed_min >= p->e_speed_max)
    return pe::fail(PE_EINVAL, "Invalid solver options");
  if ((int64_t)p->p_speeds * p->e_speeds > 65535 || p->headings > 65535 ||
      (int64_t)p->positions * p->positions > (1 << 30))
    return pe::fail(PE_EINVAL, "Invalid solver options: grid too large");
  return PE_OK;
}

inline pe::Rel5Grid make_grid(const pe_relative_params *p) {
  pe::Rel5Grid g{};
  const double pi = std::acos(-1.0);
  g.nx = p->positions;
  g.nh = p->headings;
  g.nvp = p->p_speeds;
  g.nve = p->e_speeds;
  g.order = p->order;
  g.xp = (g.nx + 3) / 4 * 4;  // rows padded to 16 bytes
  g.sy = g.xp;
  g.sp = (int64_t)g.nx * g.xp;
  g.se = g.sp * g.nh;
  g.sv = g.se * g.nve;
  g.n_padded = g.sv * g.nvp;
  g.n = (int64_t)g.nx * g.nx * g.nh * g.nve * g.nvp;
  g.extent = p->extent;
  g.dx = 2 * p->extent / (p->positions - 1);
  g.dphi = 2 * pi / p->headings;
  g.dvp = (p->p_speed_max - p->p_speed_min) / (p->p_speeds - 1);
  g.dve = (p->e_speed_max - p->e_speed_min) / (p->e_speeds - 1);
  g.vp_lo = p->p_speed_min;
  g.ve_lo = p->e_speed_min;
  g.acc_p = p->p_acceleration;
  g.acc_e = p->e_acceleration;
  g.curv_p = p->p_curvature;
  g.curv_e = p->e_curvature;
  pe::set_reciprocals(g);
  return g;
}

inline double cfl_limit(const pe_relative_params *p, const pe::Rel5Grid &g) {
  const double VP = std::max(std::abs(p->p_speed_min), std::abs(p->p_speed_max));
  const double VE = std::max(std::abs(p->e_speed_min), std::abs(p->e_speed_max));
  const double rate = (VP + VE + VP * p->p_curvature * p->extent) / g.dx +
                      (VE + VP * p->p_curvature * p->extent) / g.dx +
                      (VP * p->p_curvature + VE * p->e_curvature) / g.dphi +
                      p->p_acceleration / g.dvp + p->e_acceleration / g.dve;
  return p->cfl / rate;
}

// sin / cos of the heading axis q_k = -pi + k dphi (native_relative.cpp:84-89).
inline void heading_tables(const pe::Rel5Grid &g, std::vector<double> *sn,
                           std::vector<double> *cs) {
  const double pi = std::acos(-1.0);
  sn->resize(g.nh);
  cs->resize(g.nh);
  for (int k = 0; k < g.nh; k++) {
    const double q = -pi + k * g.dphi;
    (*sn)[k] = std::sin(q);
    (*cs)[k] = std::cos(q);
  }
}

// The circular capture field float(hypot(x, y) - radius) of one (y, x)
// plane, computed in double (native_relative.cpp:91-100).
inline void capture_plane(const pe::Rel5Grid &g, double radius, float *plane) {
  for (int iy = 0; iy < g.nx; iy++) {
    const double y = -g.extent + iy * g.dx;
    for (int ix = 0; ix < g.nx; ix++)
      plane[(size_t)iy * g.nx + ix] = (float)(std::hypot(-g.extent + ix * g.dx, y) - radius);
  }
}

}  // namespace rel5host
}  // namespace pe
