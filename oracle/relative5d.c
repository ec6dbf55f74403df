/*
 * CPU ORACLE — test infrastructure only.  Nothing in the product links this
 * file: only tests/, the smoke check and bench.py's CPU-baseline leg load the
 * shared library built from it (oracle/_build/liboracle.so).
 *
 * Restatement of the reference's relative 5D ENO/Lax-Friedrichs capture-tube
 * update, pursuit-evasion-core src/pursuit_evasion/reversible/native_relative.cpp:
 *   - grid spacings and CFL limit        native_relative.cpp:70-81
 *   - circular-capture initial field     native_relative.cpp:91-100
 *   - ENO1/ENO2 one-axis slopes          native_relative.cpp:38-67
 *   - Isaacs Hamiltonian + LF + update   native_relative.cpp:124-172
 *   - frame/step driver                  native_relative.cpp:173-207
 *
 * Two storage modes:
 *   po_rel_stage_f32 : float32 storage, double local arithmetic.  The
 *       operations are evaluated in the same order as the reference so that a
 *       non-contracting x86-64 build reproduces the reference executable bit
 *       for bit (checked by tests/test_oracle.py against the executable and
 *       its golden vectors).
 *   po_rel_stage_f64 : double storage, the "FP64 oracle" used to report the
 *       max-abs error of float32-storage tables.
 *
 * Build with -ffp-contract=off: fused multiply-adds would change the bits.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"


typedef struct {
  double dx, dphi, dvp, dve;
  size_t sy, sp, se, sv, n;
} po_rel_geom;

static po_rel_geom geom_of(const po_rel_cfg *c) {
  po_rel_geom g;
  const double pi = acos(-1.0);
  g.dx = 2 * c->extent / (c->nx - 1);
  g.dphi = 2 * pi / c->nh;
  g.dvp = (c->vp_hi - c->vp_lo) / (c->nvp - 1);
  g.dve = (c->ve_hi - c->ve_lo) / (c->nve - 1);
  g.sy = (size_t)c->nx;
  g.sp = (size_t)c->nx * c->nx;
  g.se = g.sp * c->nh;
  g.sv = g.se * c->nve;
  g.n = g.sv * c->nvp;
  return g;
}

size_t po_rel_cells(const po_rel_cfg *c) { return geom_of(c).n; }

double po_rel_cfl_limit(const po_rel_cfg *c) {
  const po_rel_geom g = geom_of(c);
  const double VP = fmax(fabs(c->vp_lo), fabs(c->vp_hi));
  const double VE = fmax(fabs(c->ve_lo), fabs(c->ve_hi));
  const double rate = (VP + VE + VP * c->curv_p * c->extent) / g.dx +
                      (VE + VP * c->curv_p * c->extent) / g.dx +
                      (VP * c->curv_p + VE * c->curv_e) / g.dphi +
                      c->acc_p / g.dvp + c->acc_e / g.dve;
  return c->cfl / rate;
}

void po_rel_init(const po_rel_cfg *c, float *field, float *arrival) {
  const po_rel_geom g = geom_of(c);
  const size_t rows = g.n / c->nx;
#pragma omp parallel for schedule(static)
  for (size_t row = 0; row < rows; row++) {
    const double y = -c->extent + (double)(row % c->nx) * g.dx;
    for (int ix = 0; ix < c->nx; ix++) {
      const size_t j = row * c->nx + ix;
      field[j] = (float)(hypot(-c->extent + ix * g.dx, y) - c->radius);
      if (arrival) arrival[j] = field[j] <= 0 ? 0.0f : NAN;
    }
  }
}

void po_rel_init_f64(const po_rel_cfg *c, double *field) {
  const po_rel_geom g = geom_of(c);
  const size_t rows = g.n / c->nx;
#pragma omp parallel for schedule(static)
  for (size_t row = 0; row < rows; row++) {
    const double y = -c->extent + (double)(row % c->nx) * g.dx;
    for (int ix = 0; ix < c->nx; ix++)
      field[row * c->nx + ix] = hypot(-c->extent + ix * g.dx, y) - c->radius;
  }
}

/* Backward/forward ENO slopes along one axis.  T is float or double storage;
 * the arithmetic is double either way.  Ghost reads wrap on a periodic axis;
 * a non-periodic axis uses a one-sided first difference at its two end nodes
 * and falls back to the centred second difference next to them. */
#define PO_DEFINE_SLOPES(NAME, T)                                               \
  static inline void NAME(const T *s, size_t j, size_t stride, int pos, int n, \
                          double h, int periodic, int order, double *lo,       \
                          double *hi) {                                         \
    const double v = s[j];                                                     \
    ptrdiff_t off_m1 = -1, off_p1 = 1, off_m2 = -2, off_p2 = 2;                \
    if (periodic) {                                                            \
      off_m1 = (pos - 1 < 0) ? n - 1 : -1;                                     \
      off_p1 = (pos + 1 >= n) ? 1 - n : 1;                                     \
      off_m2 = (pos - 2 < 0) ? n - 2 : -2;                                     \
      off_p2 = (pos + 2 >= n) ? 2 - n : 2;                                     \
    } else if (pos == 0) {                                                     \
      *lo = *hi = ((double)s[j + stride] - v) / h;                             \
      return;                                                                  \
    } else if (pos == n - 1) {                                                 \
      *lo = *hi = (v - (double)s[j - stride]) / h;                             \
      return;                                                                  \
    }                                                                          \
    const double vm = s[(ptrdiff_t)j + off_m1 * (ptrdiff_t)stride];           \
    const double vp = s[(ptrdiff_t)j + off_p1 * (ptrdiff_t)stride];           \
    double l = (v - vm) / h, r = (vp - v) / h;                                 \
    if (order == 2) {                                                          \
      const double hh = h * h;                                                 \
      const double c2 = (vp - 2 * v + vm) / hh;                                \
      double l2 = c2, r2 = c2;                                                 \
      if (periodic || pos >= 2)                                                \
        l2 = (v - 2 * vm +                                                     \
              (double)s[(ptrdiff_t)j + off_m2 * (ptrdiff_t)stride]) / hh;      \
      if (periodic || pos + 2 < n)                                             \
        r2 = ((double)s[(ptrdiff_t)j + off_p2 * (ptrdiff_t)stride] - 2 * vp + \
              v) / hh;                                                         \
      l += .5 * h * (fabs(l2) < fabs(c2) ? l2 : c2);                           \
      r -= .5 * h * (fabs(c2) < fabs(r2) ? c2 : r2);                           \
    }                                                                          \
    *lo = l;                                                                   \
    *hi = r;                                                                   \
  }

PO_DEFINE_SLOPES(slopes_f32, float)
PO_DEFINE_SLOPES(slopes_f64, double)

/* Isaacs Hamiltonian of the relative game plus local Lax-Friedrichs
 * dissipation at one node, from its ten one-sided slopes.  The pursuer
 * minimises, the evader maximises; curvature enters through |speed|, and a
 * speed bound removes the outward acceleration. */
static inline double hamiltonian(double x, double y, double bx, double by,
                                 double wp, double we, double acc_p,
                                 double acc_e, int p_at_lo, int p_at_hi,
                                 int e_at_lo, int e_at_hi, const double *m,
                                 const double *p) {
  /* m/p order: x, y, psi, vP, vE */
  const double gx = .5 * (m[0] + p[0]), gy = .5 * (m[1] + p[1]),
               gp = .5 * (m[2] + p[2]), gv = .5 * (m[3] + p[3]),
               ge = .5 * (m[4] + p[4]);
  const double pl = p_at_lo ? 0 : -acc_p, ph = p_at_hi ? 0 : acc_p;
  const double el = e_at_lo ? 0 : -acc_e, eh = e_at_hi ? 0 : acc_e;
  const double pv_lo = pl * gv, pv_hi = ph * gv;
  const double ev_lo = el * ge, ev_hi = eh * ge;
  const double p_best = (pv_hi < pv_lo) ? pv_hi : pv_lo;
  const double e_best = (ev_lo < ev_hi) ? ev_hi : ev_lo;
  double H = bx * gx + by * gy - wp * fabs(y * gx - x * gy - gp) +
             we * fabs(gp) + p_best + e_best;
  H += .5 * ((fabs(bx) + wp * fabs(y)) * (p[0] - m[0]) +
             (fabs(by) + wp * fabs(x)) * (p[1] - m[1]) +
             (wp + we) * (p[2] - m[2]) + acc_p * (p[3] - m[3]) +
             acc_e * (p[4] - m[4]));
  return H;
}

int po_rel_stage_f32(const po_rel_cfg *c, const float *src, float *dst,
                     float *arrival, double dt, double t, int blend,
                     double *max_increase) {
  const po_rel_geom g = geom_of(c);
  const size_t rows = g.n / c->nx;
  double *sn = (double *)malloc(sizeof(double) * c->nh);
  double *cs = (double *)malloc(sizeof(double) * c->nh);
  for (int k = 0; k < c->nh; k++) {
    const double q = -acos(-1.0) + k * g.dphi;
    sn[k] = sin(q);
    cs[k] = cos(q);
  }
  double increase = 0;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(max : increase) reduction(| : bad)
  for (size_t row = 0; row < rows; row++) {
    const int iy = (int)(row % c->nx);
    const int ip = (int)((row / c->nx) % c->nh);
    const int ie = (int)((row / ((size_t)c->nx * c->nh)) % c->nve);
    const int iv = (int)(row / ((size_t)c->nx * c->nh * c->nve));
    const double y = -c->extent + iy * g.dx;
    const double vp = c->vp_lo + iv * g.dvp, ve = c->ve_lo + ie * g.dve;
    const double wp = fabs(vp) * c->curv_p, we = fabs(ve) * c->curv_e;
    const double bx = ve * cs[ip] - vp, by = ve * sn[ip];
    for (int ix = 0; ix < c->nx; ix++) {
      const size_t j = row * c->nx + ix;
      const double x = -c->extent + ix * g.dx;
      double m[5], p[5];
      slopes_f32(src, j, 1, ix, c->nx, g.dx, 0, c->order, &m[0], &p[0]);
      slopes_f32(src, j, g.sy, iy, c->nx, g.dx, 0, c->order, &m[1], &p[1]);
      slopes_f32(src, j, g.sp, ip, c->nh, g.dphi, 1, c->order, &m[2], &p[2]);
      slopes_f32(src, j, g.sv, iv, c->nvp, g.dvp, 0, c->order, &m[3], &p[3]);
      slopes_f32(src, j, g.se, ie, c->nve, g.dve, 0, c->order, &m[4], &p[4]);
      const double H =
          hamiltonian(x, y, bx, by, wp, we, c->acc_p, c->acc_e, iv == 0,
                      iv == c->nvp - 1, ie == 0, ie == c->nve - 1, m, p);
      const double old = src[j];
      const double prev = blend ? (double)dst[j] : old;
      double value = old + dt * (H < 0. ? H : 0.);
      if (blend) value = .5 * (prev + value);
      if (!isfinite(value)) {
        bad = 1;
        continue;
      }
      dst[j] = (float)value;
      const double inc = (double)dst[j] - prev;
      if (inc > increase) increase = inc;
      if (arrival && (blend || c->order == 1) && prev > 0 && dst[j] <= 0 &&
          isnan(arrival[j]))
        arrival[j] = (float)(t + dt * prev / (prev - (double)dst[j]));
    }
  }
  free(sn);
  free(cs);
  if (max_increase) *max_increase = increase;
  return bad ? PO_ENONFINITE : 0;
}

int po_rel_stage_f64(const po_rel_cfg *c, const double *src, double *dst,
                     double dt, int blend) {
  const po_rel_geom g = geom_of(c);
  const size_t rows = g.n / c->nx;
  double *sn = (double *)malloc(sizeof(double) * c->nh);
  double *cs = (double *)malloc(sizeof(double) * c->nh);
  for (int k = 0; k < c->nh; k++) {
    const double q = -acos(-1.0) + k * g.dphi;
    sn[k] = sin(q);
    cs[k] = cos(q);
  }
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (size_t row = 0; row < rows; row++) {
    const int iy = (int)(row % c->nx);
    const int ip = (int)((row / c->nx) % c->nh);
    const int ie = (int)((row / ((size_t)c->nx * c->nh)) % c->nve);
    const int iv = (int)(row / ((size_t)c->nx * c->nh * c->nve));
    const double y = -c->extent + iy * g.dx;
    const double vp = c->vp_lo + iv * g.dvp, ve = c->ve_lo + ie * g.dve;
    const double wp = fabs(vp) * c->curv_p, we = fabs(ve) * c->curv_e;
    const double bx = ve * cs[ip] - vp, by = ve * sn[ip];
    for (int ix = 0; ix < c->nx; ix++) {
      const size_t j = row * c->nx + ix;
      const double x = -c->extent + ix * g.dx;
      double m[5], p[5];
      slopes_f64(src, j, 1, ix, c->nx, g.dx, 0, c->order, &m[0], &p[0]);
      slopes_f64(src, j, g.sy, iy, c->nx, g.dx, 0, c->order, &m[1], &p[1]);
      slopes_f64(src, j, g.sp, ip, c->nh, g.dphi, 1, c->order, &m[2], &p[2]);
      slopes_f64(src, j, g.sv, iv, c->nvp, g.dvp, 0, c->order, &m[3], &p[3]);
      slopes_f64(src, j, g.se, ie, c->nve, g.dve, 0, c->order, &m[4], &p[4]);
      const double H =
          hamiltonian(x, y, bx, by, wp, we, c->acc_p, c->acc_e, iv == 0,
                      iv == c->nvp - 1, ie == 0, ie == c->nve - 1, m, p);
      const double old = src[j];
      const double prev = blend ? dst[j] : old;
      double value = old + dt * (H < 0. ? H : 0.);
      if (blend) value = .5 * (prev + value);
      if (!isfinite(value)) bad = 1;
      dst[j] = value;
    }
  }
  free(sn);
  free(cs);
  return bad ? PO_ENONFINITE : 0;
}

/* Frame/step driver of the reference executable: frames at
 * min(k*output_dt, horizon), internal steps of min(cfl_limit, goal - t). */
int po_rel_solve_f32(const po_rel_cfg *c, double horizon, double output_dt,
                     float *frames, float *arrival, long *steps_out) {
  const po_rel_geom g = geom_of(c);
  const double limit = po_rel_cfl_limit(c);
  float *a = (float *)malloc(sizeof(float) * g.n);
  float *b = (float *)malloc(sizeof(float) * g.n);
  if (!a || !b) {
    free(a);
    free(b);
    return PO_ENOMEM;
  }
  po_rel_init(c, a, arrival);
  memcpy(frames, a, sizeof(float) * g.n);
  const int outputs = (int)ceil(horizon / output_dt - 1e-10);
  double t = 0;
  long steps = 0;
  int rc = 0;
  for (int out = 1; out <= outputs && rc == 0; out++) {
    const double goal = fmin(horizon, out * output_dt);
    while (t < goal - 1e-12 && rc == 0) {
      const double dt = fmin(limit, goal - t);
      if (c->order == 1) {
        rc = po_rel_stage_f32(c, a, b, arrival, dt, t, 0, NULL);
        float *s = a;
        a = b;
        b = s;
      } else {
        rc = po_rel_stage_f32(c, a, b, arrival, dt, t, 0, NULL);
        if (rc == 0) rc = po_rel_stage_f32(c, b, a, arrival, dt, t, 1, NULL);
      }
      t += dt;
      steps++;
    }
    memcpy(frames + (size_t)out * g.n, a, sizeof(float) * g.n);
  }
  if (steps_out) *steps_out = steps;
  free(a);
  free(b);
  return rc;
}

int po_rel_solve_f64(const po_rel_cfg *c, double horizon, double output_dt,
                     double *final, long *steps_out) {
  const po_rel_geom g = geom_of(c);
  const double limit = po_rel_cfl_limit(c);
  double *b = (double *)malloc(sizeof(double) * g.n);
  if (!b) return PO_ENOMEM;
  po_rel_init_f64(c, final);
  const int outputs = (int)ceil(horizon / output_dt - 1e-10);
  double t = 0;
  long steps = 0;
  int rc = 0;
  for (int out = 1; out <= outputs && rc == 0; out++) {
    const double goal = fmin(horizon, out * output_dt);
    while (t < goal - 1e-12 && rc == 0) {
      const double dt = fmin(limit, goal - t);
      rc = po_rel_stage_f64(c, final, b, dt, 0);
      if (rc == 0) {
        if (c->order == 1)
          memcpy(final, b, sizeof(double) * g.n);
        else
          rc = po_rel_stage_f64(c, b, final, dt, 1);
      }
      t += dt;
      steps++;
    }
  }
  if (steps_out) *steps_out = steps;
  free(b);
  return rc;
}
