/*
 * CPU ORACLE — test infrastructure only (see relative5d.c for the rules).
 *
 * Restatement of the reference's legacy six-dimensional square game,
 * pursuit-evasion-core src/pursuit_evasion/dp/native_square.cpp:
 *   - spacings, axes and the dt bound          native_square.cpp:87-103
 *   - target (capture or evader fault) and
 *     avoid (pursuer fault) surfaces           native_square.cpp:110-128
 *   - ENO1/ENO2 slopes with signed linear
 *     extrapolation beyond the box             native_square.cpp:31-62
 *   - one stage of the RK1/RK2 update, tube
 *     minimum and avoid floor, arrival         native_square.cpp:145-183
 * Storage order [xP, yP, thP, xE, yE, thE], thE fastest; float32 fields and
 * float32 local arithmetic in the reference's order (no FMA), so a baseline
 * x86-64 build reproduces the reference executable bit for bit (pinned by
 * tests/golden/square6d_*.npz, made by that executable).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#include "oracle.h"

typedef struct {
  int shape[6];
  size_t stride[6];
  size_t n;
  float dx, dh;
  float *x, *cs, *sn;
} s6_geom;

static void s6_make(const po_s6_cfg *c, s6_geom *g) {
  const double pi = acos(-1.0);
  g->dx = 2 * c->extent / (c->n - 1);
  g->dh = (float)(2 * pi / c->nh);
  const int shape[6] = {c->n, c->n, c->nh, c->n, c->n, c->nh};
  for (int k = 0; k < 6; k++) g->shape[k] = shape[k];
  g->stride[5] = 1;
  for (int k = 4; k >= 0; k--) g->stride[k] = g->stride[k + 1] * shape[k + 1];
  g->n = g->stride[0] * c->n;
  g->x = (float *)malloc(sizeof(float) * c->n);
  g->cs = (float *)malloc(sizeof(float) * c->nh);
  g->sn = (float *)malloc(sizeof(float) * c->nh);
  for (int i = 0; i < c->n; i++) g->x[i] = -c->extent + i * g->dx;
  for (int i = 0; i < c->nh; i++) {
    g->cs[i] = (float)cos(-pi + i * 2 * pi / c->nh);
    g->sn[i] = (float)sin(-pi + i * 2 * pi / c->nh);
  }
}

static void s6_free(s6_geom *g) {
  free(g->x);
  free(g->cs);
  free(g->sn);
}

size_t po_s6_cells(const po_s6_cfg *c) {
  return (size_t)c->n * c->n * c->nh * c->n * c->n * c->nh;
}

double po_s6_dt_limit(const po_s6_cfg *c) {
  const double pi = acos(-1.0);
  const float dx = 2 * c->extent / (c->n - 1), dh = (float)(2 * pi / c->nh);
  return c->cfl / (2 * (c->vp + c->ve) / (double)dx + (c->wp + c->we) / (double)dh);
}

static inline void s6_index(const s6_geom *g, size_t j, int q[6]) {
  for (int k = 0; k < 6; k++) q[k] = (int)((j / g->stride[k]) % g->shape[k]);
}

void po_s6_init(const po_s6_cfg *c, float *a, float *arrival) {
  s6_geom g;
  s6_make(c, &g);
  const size_t blocks = g.n / c->nh;
#pragma omp parallel for schedule(static)
  for (size_t block = 0; block < blocks; block++) {
    int q[6];
    s6_index(&g, block * c->nh, q);
    const float capture = hypotf(g.x[q[0]] - g.x[q[3]], g.x[q[1]] - g.x[q[4]]) - c->radius;
    const float e_fault = c->arena - fmaxf(fabsf(g.x[q[3]]), fabsf(g.x[q[4]]));
    const float target = e_fault < capture ? e_fault : capture;
    const float avoid = fmaxf(fabsf(g.x[q[0]]), fabsf(g.x[q[1]])) - c->arena + 1e-6f;
    const float initial = target < avoid ? avoid : target;
    for (int k = 0; k < c->nh; k++) {
      a[block * c->nh + k] = initial;
      arrival[block * c->nh + k] = initial <= 0 ? 0.0f : NAN;
    }
  }
  s6_free(&g);
}

/* Value beyond a non-periodic end: the end value pushed away from zero by
 * the end difference, once per missing node; periodic axes wrap. */
static inline float s6_at(const float *v, size_t j, size_t stride, int pos, int n,
                          int offset, int periodic) {
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

static inline void s6_slopes(const float *v, size_t j, size_t stride, int pos, int n, float h,
                             int periodic, int order, float *left, float *right) {
  const float f = v[j];
  const float fm = s6_at(v, j, stride, pos, n, -1, periodic);
  const float fp = s6_at(v, j, stride, pos, n, 1, periodic);
  *left = (f - fm) / h;
  *right = (fp - f) / h;
  if (order == 2) {
    const float dl = (f - 2 * fm + s6_at(v, j, stride, pos, n, -2, periodic)) / (h * h);
    const float dc = (fp - 2 * f + fm) / (h * h);
    const float dr = (s6_at(v, j, stride, pos, n, 2, periodic) - 2 * fp + f) / (h * h);
    const float a = fabsf(dl) <= fabsf(dc) ? dl : dc;
    const float b = fabsf(dc) <= fabsf(dr) ? dc : dr;
    *left += .5f * h * a;
    *right -= .5f * h * b;
  }
}

int po_s6_stage(const po_s6_cfg *c, const float *src, float *dst, const float *base,
                float *arrival, float dt, double tau) {
  s6_geom g;
  s6_make(c, &g);
  const size_t blocks = g.n / c->nh;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (size_t block = 0; block < blocks; block++) {
    int q[6];
    s6_index(&g, block * c->nh, q);
    for (int eh = 0; eh < c->nh; eh++) {
      const size_t j = block * c->nh + eh;
      q[5] = eh;
      const float f[6] = {c->vp * g.cs[q[2]], c->vp * g.sn[q[2]], 0,
                          c->ve * g.cs[q[5]], c->ve * g.sn[q[5]], 0};
      float gr[6], diss = 0, H = 0;
      for (int k = 0; k < 6; k++) {
        float lm, rp;
        const int periodic = k == 2 || k == 5;
        s6_slopes(src, j, g.stride[k], q[k], g.shape[k], periodic ? g.dh : g.dx, periodic,
                  c->order, &lm, &rp);
        gr[k] = (lm + rp) * .5f;
        const float alpha = k == 2 ? c->wp : k == 5 ? c->we : fabsf(f[k]);
        diss += alpha * (rp - lm) * .5f;
        H += f[k] * gr[k];
      }
      H += -c->wp * fabsf(gr[2]) + c->we * fabsf(gr[5]);
      float value = src[j] + dt * (H + diss);
      if (base) value = .5f * (base[j] + value);
      if (c->order == 1 || base) {
        const float previous = base ? base[j] : src[j];
        const float avoid = fmaxf(fabsf(g.x[q[0]]), fabsf(g.x[q[1]])) - c->arena + 1e-6f;
        /* std::max(std::min(value, previous), avoid) */
        const float tube = previous < value ? previous : value;
        value = tube < avoid ? avoid : tube;
        if (arrival && previous > 0 && value <= 0 && isnan(arrival[j]))
          arrival[j] = (float)tau + dt * previous / (previous - value);
      }
      if (!isfinite(value)) bad = 1;
      dst[j] = value;
    }
  }
  s6_free(&g);
  return bad ? PO_ENONFINITE : 0;
}
