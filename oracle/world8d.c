/*
 * CPU ORACLE — test infrastructure only (see relative5d.c for the rules).
 *
 * Restatement of the reference's dense 8D ENO/LF capture step,
 * pursuit-evasion-core src/pursuit_evasion/reversible/native_world.cpp:
 *   - float32 spacings, axes and dt bound     native_world.cpp:122-150
 *   - square-arena target/avoid surfaces      native_world.cpp:155-176
 *   - ENO slopes with signed extrapolation
 *     and the inward speed boundary           native_world.cpp:32-74
 *   - one stage of the RK1/RK2 update         native_world.cpp:261-314
 * plus the exact oriented-rectangle separating-axis contact value of
 * src/pursuit_evasion/local_game/geometry.py:15-36 as the capture field.
 *
 * Storage order [xP, yP, thP, vP, xE, yE, thE, vE], vE fastest.  Arithmetic is
 * float32 like the reference, evaluated in the reference's order (no FMA), so a
 * baseline x86-64 build reproduces the reference executable bit for bit.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#include "oracle.h"

typedef struct {
  int shape[8];
  size_t stride[8];
  float spacing[8];
  size_t n;
  float *x, *cs, *sn, *pv, *ev;
} w8_geom;

static void w8_make(const po_w8_cfg *c, w8_geom *g) {
  const double pi = acos(-1.0);
  const float dx = 2 * c->extent / (c->n - 1);
  const float dh = (float)(2 * pi / c->nh);
  const float dvp = (c->p_hi - c->p_lo) / (c->np - 1);
  const float dve = (c->e_hi - c->e_lo) / (c->ne - 1);
  const int shape[8] = {c->n, c->n, c->nh, c->np, c->n, c->n, c->nh, c->ne};
  const float spacing[8] = {dx, dx, dh, dvp, dx, dx, dh, dve};
  for (int k = 0; k < 8; k++) {
    g->shape[k] = shape[k];
    g->spacing[k] = spacing[k];
  }
  g->stride[7] = 1;
  for (int k = 6; k >= 0; k--) g->stride[k] = g->stride[k + 1] * shape[k + 1];
  g->n = g->stride[0] * c->n;
  g->x = (float *)malloc(sizeof(float) * c->n);
  g->cs = (float *)malloc(sizeof(float) * c->nh);
  g->sn = (float *)malloc(sizeof(float) * c->nh);
  g->pv = (float *)malloc(sizeof(float) * c->np);
  g->ev = (float *)malloc(sizeof(float) * c->ne);
  for (int i = 0; i < c->n; i++) g->x[i] = -c->extent + i * dx;
  for (int i = 0; i < c->nh; i++) {
    const double angle = -pi + i * 2 * pi / c->nh;
    g->cs[i] = (float)cos(angle);
    g->sn[i] = (float)sin(angle);
  }
  for (int i = 0; i < c->np; i++) g->pv[i] = c->p_lo + i * dvp;
  for (int i = 0; i < c->ne; i++) g->ev[i] = c->e_lo + i * dve;
}

static void w8_free(w8_geom *g) {
  free(g->x);
  free(g->cs);
  free(g->sn);
  free(g->pv);
  free(g->ev);
}

size_t po_w8_cells(const po_w8_cfg *c) {
  size_t n = 1;
  const int shape[8] = {c->n, c->n, c->nh, c->np, c->n, c->n, c->nh, c->ne};
  for (int k = 0; k < 8; k++) n *= (size_t)shape[k];
  return n;
}

double po_w8_dt_limit(const po_w8_cfg *c) {
  const double pi = acos(-1.0);
  const float dx = 2 * c->extent / (c->n - 1);
  const float dh = (float)(2 * pi / c->nh);
  const float dvp = (c->p_hi - c->p_lo) / (c->np - 1);
  const float dve = (c->e_hi - c->e_lo) / (c->ne - 1);
  const float pabs = fmaxf(fabsf(c->p_lo), fabsf(c->p_hi));
  const float eabs = fmaxf(fabsf(c->e_lo), fabsf(c->e_hi));
  return c->cfl / (2 * (double)(pabs + eabs) / dx +
                   (double)(pabs * c->kp + eabs * c->ke) / dh +
                   (double)c->ap / dvp + (double)c->ae / dve);
}

/* Value beyond a non-periodic end: the end value pushed away from zero by the
 * end difference, once per missing node. */
static inline float ghost(const float *v, size_t j, size_t stride, int pos,
                          int n, int offset, int periodic) {
  int q = pos + offset;
  if (periodic) {
    q = (q % n + n) % n;
    return v[(ptrdiff_t)j + (ptrdiff_t)(q - pos) * (ptrdiff_t)stride];
  }
  if (q < 0) {
    const size_t edge = j - (size_t)pos * stride;
    const float a = v[edge], b = v[edge + stride];
    return a + (-q) * fabsf(b - a) * ((a > 0) - (a < 0));
  }
  if (q >= n) {
    const size_t edge = j + (size_t)(n - 1 - pos) * stride;
    const float a = v[edge], b = v[edge - stride];
    return a + (q - n + 1) * fabsf(a - b) * ((a > 0) - (a < 0));
  }
  return v[(ptrdiff_t)j + (ptrdiff_t)offset * (ptrdiff_t)stride];
}

static inline void w8_slopes(const float *v, size_t j, size_t stride, int pos,
                             int n, float h, int periodic, int inward, int order,
                             float *lo, float *hi) {
  if (inward && pos == 0) {
    *lo = *hi = (v[j + stride] - v[j]) / h;
    return;
  }
  if (inward && pos == n - 1) {
    *lo = *hi = (v[j] - v[j - stride]) / h;
    return;
  }
  const float f = v[j];
  const float fm = ghost(v, j, stride, pos, n, -1, periodic);
  const float fp = ghost(v, j, stride, pos, n, 1, periodic);
  float l = (f - fm) / h, r = (fp - f) / h;
  if (order == 2) {
    const float dc = (fp - 2 * f + fm) / (h * h);
    const float dl =
        inward && pos < 2
            ? dc
            : (f - 2 * fm + ghost(v, j, stride, pos, n, -2, periodic)) / (h * h);
    const float dr =
        inward && pos + 2 >= n
            ? dc
            : (ghost(v, j, stride, pos, n, 2, periodic) - 2 * fp + f) / (h * h);
    l += .5f * h * (fabsf(dl) <= fabsf(dc) ? dl : dc);
    r -= .5f * h * (fabsf(dc) <= fabsf(dr) ? dc : dr);
  }
  *lo = l;
  *hi = r;
}

void po_w8_init_square(const po_w8_cfg *c, float *a, float *arrival) {
  w8_geom g;
  w8_make(c, &g);
  const size_t inner = (size_t)c->nh * c->ne;
  const size_t blocks = g.n / inner;
#pragma omp parallel for schedule(static)
  for (size_t block = 0; block < blocks; block++) {
    const size_t begin = block * inner;
    int q[8];
    for (int k = 0; k < 8; k++) q[k] = (int)((begin / g.stride[k]) % g.shape[k]);
    const float capture =
        hypotf(g.x[q[0]] - g.x[q[4]], g.x[q[1]] - g.x[q[5]]) - c->radius;
    const float e_fault = c->arena - fmaxf(fabsf(g.x[q[4]]), fabsf(g.x[q[5]]));
    const float target = e_fault < capture ? e_fault : capture;
    const float avoid =
        fmaxf(fabsf(g.x[q[0]]), fabsf(g.x[q[1]])) - c->arena + 1e-6f;
    const float initial = target < avoid ? avoid : target;
    for (size_t k = 0; k < inner; k++) {
      a[begin + k] = initial;
      if (arrival) arrival[begin + k] = initial <= 0 ? 0.0f : NAN;
    }
  }
  w8_free(&g);
}

/* Oriented-rectangle contact value (geometry.py:15-36), double precision:
 * the larger of the four separating-axis gaps; <= 0 exactly when the two
 * footprints touch or overlap. */
double po_rect_separation(double px, double py, double pth, double ex,
                          double ey, double eth, double p_len, double p_wid,
                          double e_len, double e_wid) {
  const double d0 = ex - px, d1 = ey - py;
  const double delta = eth - pth;
  const double ca = fabs(cos(delta)), sa = fabs(sin(delta));
  const double poses[2] = {pth, eth};
  const double own_l[2] = {p_len, e_len}, own_w[2] = {p_wid, e_wid};
  const double oth_l[2] = {e_len, p_len}, oth_w[2] = {e_wid, p_wid};
  double best = -INFINITY;
  for (int k = 0; k < 2; k++) {
    const double c = cos(poses[k]), s = sin(poses[k]);
    const double x = d0 * c + d1 * s;
    const double y = -d0 * s + d1 * c;
    const double gx =
        fabs(x) - own_l[k] / 2 - (oth_l[k] * ca + oth_w[k] * sa) / 2;
    const double gy =
        fabs(y) - own_w[k] / 2 - (oth_l[k] * sa + oth_w[k] * ca) / 2;
    if (gx > best) best = gx;
    if (gy > best) best = gy;
  }
  return best;
}

/* Capture field of the 8D contact game: rectangle contact value of the two
 * footprints at grid poses (double), stored as float; speeds do not enter. */
void po_w8_init_contact(const po_w8_cfg *c, double p_len, double p_wid,
                        double e_len, double e_wid, float *a, float *arrival) {
  w8_geom g;
  w8_make(c, &g);
  const double pi = acos(-1.0);
  const double dxd = 2 * (double)c->extent / (c->n - 1);
  const size_t inner = (size_t)c->ne;
  const size_t blocks = g.n / inner;
#pragma omp parallel for schedule(static)
  for (size_t block = 0; block < blocks; block++) {
    const size_t begin = block * inner;
    int q[8];
    for (int k = 0; k < 8; k++) q[k] = (int)((begin / g.stride[k]) % g.shape[k]);
    const double px = -(double)c->extent + q[0] * dxd;
    const double py = -(double)c->extent + q[1] * dxd;
    const double ex = -(double)c->extent + q[4] * dxd;
    const double ey = -(double)c->extent + q[5] * dxd;
    const double pth = -pi + q[2] * 2 * pi / c->nh;
    const double eth = -pi + q[6] * 2 * pi / c->nh;
    const float value = (float)po_rect_separation(px, py, pth, ex, ey, eth,
                                                  p_len, p_wid, e_len, e_wid);
    for (size_t k = 0; k < inner; k++) {
      a[begin + k] = value;
      if (arrival) arrival[begin + k] = value <= 0 ? 0.0f : NAN;
    }
  }
  w8_free(&g);
}

/* One stage: dst = src + dt*(H + dissipation); with base != NULL the RK2
 * average with base.  On the last stage of a step the tube minimum with the
 * previous value and the avoid floor are applied and arrival recorded. */
int po_w8_stage(const po_w8_cfg *c, const float *src, float *dst,
                const float *base, float *arrival, float dt, double tau) {
  return po_w8_stage_clear(c, src, dst, base, arrival, dt, tau, NULL);
}

/* The obstacle map game's surfaces (gpu_map_game.py:45-50): centre-distance
 * capture limited by the evader clearance, floored by the pursuer's. */
void po_w8_init_map(const po_w8_cfg *c, const float *p_clear, const float *e_clear,
                    float *a, float *arrival) {
  w8_geom g;
  w8_make(c, &g);
  const float dx = 2 * c->extent / (c->n - 1);
#pragma omp parallel for schedule(static)
  for (size_t j = 0; j < g.n; j++) {
    int q[8];
    for (int k = 0; k < 8; k++) q[k] = (int)((j / g.stride[k]) % g.shape[k]);
    const float cap = hypotf((q[0] - q[4]) * dx, (q[1] - q[5]) * dx) - c->radius;
    const float p = p_clear[((size_t)q[0] * c->n + q[1]) * c->nh + q[2]];
    const float e = e_clear[((size_t)q[4] * c->n + q[5]) * c->nh + q[6]];
    const float v = fmaxf(fminf(cap, e), -p + 1e-6f);
    a[j] = v;
    if (arrival) arrival[j] = v <= 0 ? 0.0f : NAN;
  }
  w8_free(&g);
}

/* po_w8_stage with the map game's avoid floor -p_clear[xP, yP, thP] + 1e-6
 * (gpu_map_game.py:64-66) when p_clear != NULL. */
int po_w8_stage_clear(const po_w8_cfg *c, const float *src, float *dst, const float *base,
                      float *arrival, float dt, double tau, const float *p_clear) {
  w8_geom g;
  w8_make(c, &g);
  const size_t inner = (size_t)c->nh * c->ne;
  const size_t blocks = g.n / inner;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (size_t block = 0; block < blocks; block++) {
    const size_t begin = block * inner;
    int q[8];
    for (int k = 0; k < 8; k++) q[k] = (int)((begin / g.stride[k]) % g.shape[k]);
    const float vp = g.pv[q[3]];
    const float palo = q[3] == 0 ? 0 : -c->ap;
    const float pahi = q[3] == c->np - 1 ? 0 : c->ap;
    const float fpx = vp * g.cs[q[2]], fpy = vp * g.sn[q[2]];
    const float wp = fabsf(vp) * c->kp;
    const float avoid =
        p_clear ? -p_clear[((size_t)q[0] * c->n + q[1]) * c->nh + q[2]] + 1e-6f
        : c->avoid_square
            ? fmaxf(fabsf(g.x[q[0]]), fabsf(g.x[q[1]])) - c->arena + 1e-6f
            : -INFINITY;
    for (int eh = 0; eh < c->nh; eh++) {
      q[6] = eh;
      for (int iv = 0; iv < c->ne; iv++) {
        q[7] = iv;
        const size_t j = begin + (size_t)eh * c->ne + iv;
        const float ve = g.ev[iv], we = fabsf(ve) * c->ke;
        const float ealo = iv == 0 ? 0 : -c->ae;
        const float eahi = iv == c->ne - 1 ? 0 : c->ae;
        const float flow[8] = {fpx, fpy, 0, 0, ve * g.cs[eh], ve * g.sn[eh], 0,
                               0};
        float grad[8], H = 0, diss = 0;
        for (int k = 0; k < 8; k++) {
          float lm, rp;
          w8_slopes(src, j, g.stride[k], q[k], g.shape[k], g.spacing[k],
                    k == 2 || k == 6, c->linear_speed && (k == 3 || k == 7),
                    c->order, &lm, &rp);
          grad[k] = .5f * (lm + rp);
          const float alpha = k == 2   ? wp
                              : k == 3 ? c->ap
                              : k == 6 ? we
                              : k == 7 ? c->ae
                                       : fabsf(flow[k]);
          H += flow[k] * grad[k];
          diss += .5f * alpha * (rp - lm);
        }
        const float p_lo_term = palo * grad[3], p_hi_term = pahi * grad[3];
        const float e_lo_term = ealo * grad[7], e_hi_term = eahi * grad[7];
        H += -wp * fabsf(grad[2]) + we * fabsf(grad[6]) +
             (p_hi_term < p_lo_term ? p_hi_term : p_lo_term) +
             (e_lo_term < e_hi_term ? e_hi_term : e_lo_term);
        float value = src[j] + dt * (H + diss);
        if (base) value = .5f * (base[j] + value);
        if (c->order == 1 || base) {
          const float previous = base ? base[j] : src[j];
          /* std::min(value, previous) and std::max(., avoid) semantics */
          const float tube = previous < value ? previous : value;
          value = tube < avoid ? avoid : tube;
          if (arrival && previous > 0 && value <= 0 && isnan(arrival[j]))
            arrival[j] = (float)tau + dt * previous / (previous - value);
        }
        if (!isfinite(value)) bad = 1;
        dst[j] = value;
      }
    }
  }
  w8_free(&g);
  return bad ? PO_ENONFINITE : 0;
}

/* ------------------------------------------------------------------------
 * The same stage in double precision (double fields, the float32 grid axes
 * and spacings promoted to double): the rounding-free reference against
 * which float32 variants of the step are measured.  Same formulas and
 * order as po_w8_stage. */
static inline double ghost_f64(const double *v, size_t j, size_t stride,
                               int pos, int n, int offset, int periodic) {
  int q = pos + offset;
  if (periodic) {
    q = (q % n + n) % n;
    return v[(ptrdiff_t)j + (ptrdiff_t)(q - pos) * (ptrdiff_t)stride];
  }
  if (q < 0) {
    const size_t edge = j - (size_t)pos * stride;
    const double a = v[edge], b = v[edge + stride];
    return a + (-q) * fabs(b - a) * ((a > 0) - (a < 0));
  }
  if (q >= n) {
    const size_t edge = j + (size_t)(n - 1 - pos) * stride;
    const double a = v[edge], b = v[edge - stride];
    return a + (q - n + 1) * fabs(a - b) * ((a > 0) - (a < 0));
  }
  return v[(ptrdiff_t)j + (ptrdiff_t)offset * (ptrdiff_t)stride];
}

static inline void w8_slopes_f64(const double *v, size_t j, size_t stride,
                                 int pos, int n, double h, int periodic,
                                 int inward, int order, double *lo,
                                 double *hi) {
  if (inward && pos == 0) {
    *lo = *hi = (v[j + stride] - v[j]) / h;
    return;
  }
  if (inward && pos == n - 1) {
    *lo = *hi = (v[j] - v[j - stride]) / h;
    return;
  }
  const double f = v[j];
  const double fm = ghost_f64(v, j, stride, pos, n, -1, periodic);
  const double fp = ghost_f64(v, j, stride, pos, n, 1, periodic);
  double l = (f - fm) / h, r = (fp - f) / h;
  if (order == 2) {
    const double dc = (fp - 2 * f + fm) / (h * h);
    const double dl =
        inward && pos < 2
            ? dc
            : (f - 2 * fm + ghost_f64(v, j, stride, pos, n, -2, periodic)) / (h * h);
    const double dr =
        inward && pos + 2 >= n
            ? dc
            : (ghost_f64(v, j, stride, pos, n, 2, periodic) - 2 * fp + f) / (h * h);
    l += .5 * h * (fabs(dl) <= fabs(dc) ? dl : dc);
    r -= .5 * h * (fabs(dc) <= fabs(dr) ? dc : dr);
  }
  *lo = l;
  *hi = r;
}

int po_w8_stage_f64(const po_w8_cfg *c, const double *src, double *dst,
                    const double *base, double dt) {
  w8_geom g;
  w8_make(c, &g);
  const size_t inner = (size_t)c->nh * c->ne;
  const size_t blocks = g.n / inner;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (size_t block = 0; block < blocks; block++) {
    const size_t begin = block * inner;
    int q[8];
    for (int k = 0; k < 8; k++) q[k] = (int)((begin / g.stride[k]) % g.shape[k]);
    const double vp = g.pv[q[3]];
    const double ap = c->ap, ae = c->ae;
    const double palo = q[3] == 0 ? 0 : -ap;
    const double pahi = q[3] == c->np - 1 ? 0 : ap;
    const double fpx = vp * g.cs[q[2]], fpy = vp * g.sn[q[2]];
    const double wp = fabs(vp) * c->kp;
    const double avoid =
        c->avoid_square
            ? fmax(fabs((double)g.x[q[0]]), fabs((double)g.x[q[1]])) - c->arena + 1e-6
            : -INFINITY;
    for (int eh = 0; eh < c->nh; eh++) {
      q[6] = eh;
      for (int iv = 0; iv < c->ne; iv++) {
        q[7] = iv;
        const size_t j = begin + (size_t)eh * c->ne + iv;
        const double ve = g.ev[iv], we = fabs(ve) * c->ke;
        const double ealo = iv == 0 ? 0 : -ae;
        const double eahi = iv == c->ne - 1 ? 0 : ae;
        const double flow[8] = {fpx, fpy, 0, 0, ve * g.cs[eh], ve * g.sn[eh], 0, 0};
        double grad[8], H = 0, diss = 0;
        for (int k = 0; k < 8; k++) {
          double lm, rp;
          w8_slopes_f64(src, j, g.stride[k], q[k], g.shape[k], g.spacing[k],
                        k == 2 || k == 6, c->linear_speed && (k == 3 || k == 7),
                        c->order, &lm, &rp);
          grad[k] = .5 * (lm + rp);
          const double alpha = k == 2   ? wp
                               : k == 3 ? ap
                               : k == 6 ? we
                               : k == 7 ? ae
                                        : fabs(flow[k]);
          H += flow[k] * grad[k];
          diss += .5 * alpha * (rp - lm);
        }
        const double p_lo_term = palo * grad[3], p_hi_term = pahi * grad[3];
        const double e_lo_term = ealo * grad[7], e_hi_term = eahi * grad[7];
        H += -wp * fabs(grad[2]) + we * fabs(grad[6]) +
             (p_hi_term < p_lo_term ? p_hi_term : p_lo_term) +
             (e_lo_term < e_hi_term ? e_hi_term : e_lo_term);
        double value = src[j] + dt * (H + diss);
        if (base) value = .5 * (base[j] + value);
        if (c->order == 1 || base) {
          const double previous = base ? base[j] : src[j];
          const double tube = previous < value ? previous : value;
          value = tube < avoid ? avoid : tube;
        }
        if (!isfinite(value)) bad = 1;
        dst[j] = value;
      }
    }
  }
  w8_free(&g);
  return bad ? PO_ENONFINITE : 0;
}
