// Exact relative 5D ENO/LF cell update, shared by the single-grid kernel
// (relative5d_exact.cu) and the batched kernel (relative5d_batch_exact.cu).
//
// Double local arithmetic evaluated in the order of the reference
// executable (native_relative.cpp:38-67 slopes, :124-172 stage), float32
// storage -- or, with T = double, double storage: the FP64 oracle of
// oracle/relative5d.c (po_rel_stage_f64) on the GPU, used to measure the
// error of float32-storage tables.  Every translation unit that includes this header is compiled
// with -fmad=false (no multiply-add contraction, IEEE double division), so
// each stored float equals the reference CPU's bit for bit.
#pragma once
#include "div_rn.cuh"
#include "relative5d.cuh"

namespace pe {
namespace exact {

struct Slopes {
  double lo, hi;
};

using rn::div_const;  // division by a spacing, bit for bit (div_rn.cuh)

// One-axis ENO slopes at node j (native_relative.cpp:38-67); rh, rhh are
// 1/h and 1/(h*h) rounded to nearest.
template <int ORDER, typename T>
__device__ __forceinline__ Slopes eno_axis(const T *__restrict__ s,
                                           int64_t j, int64_t stride, int pos,
                                           int n, double h, double rh, double rhh,
                                           bool periodic) {
  Slopes r;
  const double v = s[j];
  if (!periodic && pos == 0) {
    r.lo = r.hi = div_const((double)s[j + stride] - v, h, rh);
    return r;
  }
  if (!periodic && pos == n - 1) {
    r.lo = r.hi = div_const(v - (double)s[j - stride], h, rh);
    return r;
  }
  // Offsets of the neighbours, wrapped on the periodic axis.
  const int64_t wrap = (int64_t)n * stride;
  const int64_t om1 = (periodic && pos < 1) ? wrap - stride : -stride;
  const int64_t op1 = (periodic && pos + 1 >= n) ? stride - wrap : stride;
  const double vm = s[j + om1];
  const double vp = s[j + op1];
  r.lo = div_const(v - vm, h, rh);
  r.hi = div_const(vp - v, h, rh);
  if (ORDER == 1) return r;
  const double hh = h * h;
  const double c2 = div_const(vp - 2 * v + vm, hh, rhh);
  double l2 = c2, r2 = c2;
  if (periodic || pos >= 2) {
    const int64_t om2 = (periodic && pos < 2) ? wrap - 2 * stride : -2 * stride;
    l2 = div_const(v - 2 * vm + (double)s[j + om2], hh, rhh);
  }
  if (periodic || pos + 2 < n) {
    const int64_t op2 =
        (periodic && pos + 2 >= n) ? 2 * stride - wrap : 2 * stride;
    r2 = div_const((double)s[j + op2] - 2 * vp + v, hh, rhh);
  }
  r.lo += .5 * h * (fabs(l2) < fabs(c2) ? l2 : c2);
  r.hi -= .5 * h * (fabs(c2) < fabs(r2) ? c2 : r2);
  return r;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *word,
                                                  double value) {
  // Non-negative doubles order like their bit patterns.
  if (value > 0) atomicMax(word, (unsigned long long)__double_as_longlong(value));
}

// Block maximum of a non-negative double (blockDim.x = 128).
__device__ __forceinline__ double block_max(double v, double *scratch) {
  for (int off = 16; off > 0; off >>= 1)
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, scratch[w]);
  __syncthreads();
  return m;
}

// One cell of one stage: reads s.src (and s.dst for the RK2 blend), writes
// s.dst and the arrival time; accumulates the sup-norm change and the
// largest increase of the step (stage 2 / RK1 only) and flags non-finite
// updates.
template <typename T>
__device__ __forceinline__ const T *stage_src(const Rel5Stage &s);
template <>
__device__ __forceinline__ const float *stage_src<float>(const Rel5Stage &s) {
  return s.src;
}
template <>
__device__ __forceinline__ const double *stage_src<double>(const Rel5Stage &s) {
  return s.src64;
}
template <typename T>
__device__ __forceinline__ T *stage_dst(const Rel5Stage &s);
template <>
__device__ __forceinline__ float *stage_dst<float>(const Rel5Stage &s) {
  return s.dst;
}
template <>
__device__ __forceinline__ double *stage_dst<double>(const Rel5Stage &s) {
  return s.dst64;
}

template <int ORDER, int BLEND, typename T = float>
__device__ __forceinline__ void cell_update(const Rel5Grid &g, const Rel5Stage &s, int ix,
                                            int iy, int ip, int iv, int ie, int64_t j,
                                            double &change_abs, double &change_up,
                                            bool &bad) {
  constexpr bool F64 = sizeof(T) == sizeof(double);
  const T *__restrict__ src = stage_src<T>(s);
  T *__restrict__ dstp = stage_dst<T>(s);

  const double x = -g.extent + ix * g.dx;
  const double y = -g.extent + iy * g.dx;
  if (s.exit_r2 > 0 && x * x + y * y > s.exit_r2) {  // held at the exit value
    dstp[j] = (T)s.exit_r;
    change_abs = change_up = 0;
    return;
  }
  const double vp = g.vp_lo + iv * g.dvp, ve = g.ve_lo + ie * g.dve;
  const double wp = fabs(vp) * g.curv_p, we = fabs(ve) * g.curv_e;
  const double bx = ve * s.cs[ip] - vp, by = ve * s.sn[ip];

  const Slopes sx = eno_axis<ORDER, T>(src, j, 1, ix, g.nx, g.dx, g.rdx, g.rdx2, false);
  const Slopes sy = eno_axis<ORDER, T>(src, j, g.sy, iy, g.nx, g.dx, g.rdx, g.rdx2, false);
  const Slopes sp =
      eno_axis<ORDER, T>(src, j, g.sp, ip, g.nh, g.dphi, g.rdphi, g.rdphi2, true);
  const Slopes sv =
      eno_axis<ORDER, T>(src, j, g.sv, iv, g.nvp, g.dvp, g.rdvp, g.rdvp2, false);
  const Slopes se =
      eno_axis<ORDER, T>(src, j, g.se, ie, g.nve, g.dve, g.rdve, g.rdve2, false);

  const double gx = .5 * (sx.lo + sx.hi), gy = .5 * (sy.lo + sy.hi),
               gp = .5 * (sp.lo + sp.hi), gv = .5 * (sv.lo + sv.hi),
               ge = .5 * (se.lo + se.hi);
  const double pl = iv == 0 ? 0 : -g.acc_p, ph = iv == g.nvp - 1 ? 0 : g.acc_p;
  const double el = ie == 0 ? 0 : -g.acc_e, eh = ie == g.nve - 1 ? 0 : g.acc_e;
  const double pv_lo = pl * gv, pv_hi = ph * gv;
  const double ev_lo = el * ge, ev_hi = eh * ge;
  const double p_best = (pv_hi < pv_lo) ? pv_hi : pv_lo;  // std::min order
  const double e_best = (ev_lo < ev_hi) ? ev_hi : ev_lo;  // std::max order
  double H = bx * gx + by * gy - wp * fabs(y * gx - x * gy - gp) +
             we * fabs(gp) + p_best + e_best;
  H += .5 * ((fabs(bx) + wp * fabs(y)) * (sx.hi - sx.lo) +
             (fabs(by) + wp * fabs(x)) * (sy.hi - sy.lo) +
             (wp + we) * (sp.hi - sp.lo) + g.acc_p * (sv.hi - sv.lo) +
             g.acc_e * (se.hi - se.lo));

  const double old = src[j];
  const double prev = BLEND ? (double)dstp[j] : old;
  double value = old + s.dt * (H < 0. ? H : 0.);
  if (BLEND) value = .5 * (prev + value);
  if (F64) {  // double storage (po_rel_stage_f64): stored as computed, no arrival
    if (!isfinite(value)) bad = true;
    dstp[j] = (T)value;
    if (BLEND || ORDER == 1) {
      const double change = value - prev;
      change_abs = fabs(change);
      change_up = change > 0 ? change : 0;
    }
  } else if (!isfinite(value)) {
    bad = true;
  } else {
    const float stored = (float)value;
    dstp[j] = (T)stored;
    if (BLEND || ORDER == 1) {
      const double change = (double)stored - prev;
      change_abs = fabs(change);
      change_up = change > 0 ? change : 0;
      if (prev > 0 && stored <= 0 && isnan(s.arrival[j]))
        s.arrival[j] = (float)(s.t + s.dt * prev / (prev - (double)stored));
    }
  }
}

}  // namespace exact
}  // namespace pe
