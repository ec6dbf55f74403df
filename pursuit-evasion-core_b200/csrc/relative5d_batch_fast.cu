// Batched relative 5D solves with a float32 cell update: the formulas of
// the exact update (native_relative.cpp:38-67 slopes, :124-172 stage) in
// float32 with reciprocal spacings and multiply-add contraction, like the
// single-grid float32 kernel.  Values agree with the exact path to float
// rounding except where rounding flips an ENO2 selection.
#include "relative5d_batch_impl.cuh"

namespace pe {
namespace {

struct SlopesF {
  float lo, hi;
};

__device__ __forceinline__ SlopesF eno2(const float *__restrict__ s, int64_t j, int64_t stride,
                                        int pos, int n, float h, float ih, bool periodic) {
  SlopesF r;
  const float v = s[j];
  if (!periodic && pos == 0) {
    r.lo = r.hi = (s[j + stride] - v) * ih;
    return r;
  }
  if (!periodic && pos == n - 1) {
    r.lo = r.hi = (v - s[j - stride]) * ih;
    return r;
  }
  const int64_t wrap = (int64_t)n * stride;
  const int64_t om1 = (periodic && pos < 1) ? wrap - stride : -stride;
  const int64_t op1 = (periodic && pos + 1 >= n) ? stride - wrap : stride;
  const float vm = s[j + om1], vp = s[j + op1];
  r.lo = (v - vm) * ih;
  r.hi = (vp - v) * ih;
  const float ihh = ih * ih;
  const float c2 = (vp - 2.f * v + vm) * ihh;
  float l2 = c2, r2 = c2;
  if (periodic || pos >= 2) {
    const int64_t om2 = (periodic && pos < 2) ? wrap - 2 * stride : -2 * stride;
    l2 = (v - 2.f * vm + s[j + om2]) * ihh;
  }
  if (periodic || pos + 2 < n) {
    const int64_t op2 = (periodic && pos + 2 >= n) ? 2 * stride - wrap : 2 * stride;
    r2 = (s[j + op2] - 2.f * vp + v) * ihh;
  }
  r.lo += .5f * h * (fabsf(l2) < fabsf(c2) ? l2 : c2);
  r.hi -= .5f * h * (fabsf(c2) < fabsf(r2) ? c2 : r2);
  return r;
}

struct FastCell {
  template <int BLEND>
  __device__ static void update(const Rel5Grid &g, const Rel5Stage &s, int ix, int iy, int ip,
                                int iv, int ie, int64_t j, double &change_abs,
                                double &change_up, bool &bad) {
    const float *__restrict__ src = s.src;
    const float dx = (float)g.dx, dphi = (float)g.dphi, dvp = (float)g.dvp, dve = (float)g.dve;
    const float ihx = 1.f / dx, ihp = 1.f / dphi, ihv = 1.f / dvp, ihe = 1.f / dve;
    const float x = (float)(-g.extent + ix * g.dx), y = (float)(-g.extent + iy * g.dx);
    const float vp = (float)(g.vp_lo + iv * g.dvp), ve = (float)(g.ve_lo + ie * g.dve);
    const float wp = fabsf(vp) * (float)g.curv_p, we = fabsf(ve) * (float)g.curv_e;
    const float bx = ve * (float)s.cs[ip] - vp, by = ve * (float)s.sn[ip];
    const SlopesF sx = eno2(src, j, 1, ix, g.nx, dx, ihx, false);
    const SlopesF sy = eno2(src, j, g.sy, iy, g.nx, dx, ihx, false);
    const SlopesF sp = eno2(src, j, g.sp, ip, g.nh, dphi, ihp, true);
    const SlopesF sv = eno2(src, j, g.sv, iv, g.nvp, dvp, ihv, false);
    const SlopesF se = eno2(src, j, g.se, ie, g.nve, dve, ihe, false);
    const float gx = .5f * (sx.lo + sx.hi), gy = .5f * (sy.lo + sy.hi),
                gp = .5f * (sp.lo + sp.hi), gv = .5f * (sv.lo + sv.hi),
                ge = .5f * (se.lo + se.hi);
    const float ap = (float)g.acc_p, ae = (float)g.acc_e;
    const float pl = iv == 0 ? 0.f : -ap, ph = iv == g.nvp - 1 ? 0.f : ap;
    const float el = ie == 0 ? 0.f : -ae, eh = ie == g.nve - 1 ? 0.f : ae;
    const float p_best = fminf(pl * gv, ph * gv);
    const float e_best = fmaxf(el * ge, eh * ge);
    float H = bx * gx + by * gy - wp * fabsf(y * gx - x * gy - gp) + we * fabsf(gp) + p_best +
              e_best;
    H += .5f * ((fabsf(bx) + wp * fabsf(y)) * (sx.hi - sx.lo) +
                (fabsf(by) + wp * fabsf(x)) * (sy.hi - sy.lo) + (wp + we) * (sp.hi - sp.lo) +
                ap * (sv.hi - sv.lo) + ae * (se.hi - se.lo));
    const float old = src[j];
    const float prev = BLEND ? s.dst[j] : old;
    float value = old + (float)s.dt * fminf(H, 0.f);
    if (BLEND) value = .5f * (prev + value);
    if (!isfinite(value)) {
      bad = true;
      return;
    }
    s.dst[j] = value;
    if (BLEND) {
      const double change = (double)value - (double)prev;
      change_abs = fabs(change);
      change_up = change > 0 ? change : 0;
      if (prev > 0.f && value <= 0.f && isnan(s.arrival[j]))
        s.arrival[j] = (float)(s.t + s.dt * (double)prev / ((double)prev - (double)value));
    }
  }
};

}  // namespace

int rel5_batch_grid_fast() { return batch_impl::grid_size<FastCell>(); }

cudaError_t rel5_batch_run_fast(const Rel5BatchArgs &args, int grid, cudaStream_t stream) {
  return batch_impl::launch<FastCell>(args, grid, stream);
}

}  // namespace pe
