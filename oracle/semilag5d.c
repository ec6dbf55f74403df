/*
 * CPU ORACLE — test infrastructure only (see relative5d.c for the rules).
 *
 * FP64 semi-Lagrangian min-max backup of the relative 5D game.  The
 * reference has no 5D semi-Lagrangian solver; this restates the pieces it
 * does have and composes them:
 *   - exact held-command arcs with speed saturation
 *       src/pursuit_evasion/reversible/model.py:86-153
 *     (integrated_speed, vehicle_step), composed with relative_state
 *       model.py:156-183 for the relative successor;
 *   - the 3x3 action catalogue product([-A,0,A],[-K,0,K]), index 3*ia+ik
 *       reversible/controllers.py:19-27;
 *   - min over pursuer actions of max over evader actions, starting the
 *     minimum at the current value (the tube minimum)
 *       local_game/grid_game.py:218-230;
 *   - multilinear interpolation over [vP, vE, psi, y, x] with periodic psi
 *       reversible/relative_table.py:76-102, linearly extrapolated beyond
 *     the position box (the ENO solver's one-sided linear extrapolation);
 *   - tie rules of the action choice: pursuer min(tied, key=(|k|,|a|,idx))
 *     with atol 1e-7 (controllers.py:122-126); evader neutral-first order
 *     (reversible/map_game_policy.py:12-18).
 *
 * Two value functionals:
 *   PO_SL_TUBE    V' = min(V, min_u max_w V(s'(u,w)))  (capture by horizon)
 *   PO_SL_MINTIME u' = 0 if the state is captured, else
 *                      (1 - b) + b * min_u max_w u(s'(u,w)),  b = exp(-dt)
 *                 the discounted (Kruzkov) minimum capture time
 *                 u = 1 - exp(-T); the interpolated value is clamped to
 *                 [0, 1].
 * Parity: unpinned by reference tests (no reference 5D semi-Lagrangian
 * solver exists); pieces are pinned as listed in tests/test_semilag_oracle.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* Exact held-acceleration speed and signed distance (model.py:86-109). */
void po_sl_integrated_speed(double v, double a, double dt, double vmin,
                            double vmax, double *v_out, double *dist) {
  const double target = a >= 0 ? vmax : vmin;
  const double hit = fabs(a) > 1e-14 ? (target - v) / a : INFINITY;
  const double active = fmin(dt, fmax(0.0, hit));
  double final = v + a * dt;
  final = final < vmin ? vmin : (final > vmax ? vmax : final);
  *v_out = final;
  *dist = v * active + 0.5 * a * active * active + final * (dt - active);
}

/* Constant-curvature arc over signed distance d with curvature k:
 * chord and turn (model.py:144-146; np.sinc(t/2pi) = sin(t/2)/(t/2)). */
static void arc(double d, double k, double *chord, double *turn) {
  const double t = k * d;
  const double half = 0.5 * t;
  *turn = t;
  *chord = fabs(half) < 1e-12 ? d : d * sin(half) / half;
}

static double wrap(double a) {
  const double two_pi = 2 * acos(-1.0);
  double r = fmod(a + acos(-1.0), two_pi);
  if (r < 0) r += two_pi;
  return r - acos(-1.0);
}

void po_sl_successor(const po_sl_cfg *c, double x, double y, double psi,
                     double vp, double ve, int up, int ue, double out[5]) {
  const double ap = (up / 3 - 1) * c->acc_p, kp = (up % 3 - 1) * c->curv_p;
  const double ae = (ue / 3 - 1) * c->acc_e, ke = (ue % 3 - 1) * c->curv_e;
  double vp2, dp, ve2, de, chp, tp, che, te;
  po_sl_integrated_speed(vp, ap, c->dt, c->vp_lo, c->vp_hi, &vp2, &dp);
  po_sl_integrated_speed(ve, ae, c->dt, c->ve_lo, c->ve_hi, &ve2, &de);
  arc(dp, kp, &chp, &tp);
  arc(de, ke, &che, &te);
  /* pursuer from the origin with heading 0, evader at (x, y) heading psi */
  const double px = chp * cos(0.5 * tp), py = chp * sin(0.5 * tp);
  const double ex = x + che * cos(psi + 0.5 * te), ey = y + che * sin(psi + 0.5 * te);
  const double dx = ex - px, dy = ey - py;
  const double cth = cos(tp), sth = sin(tp);
  out[0] = cth * dx + sth * dy;
  out[1] = -sth * dx + cth * dy;
  out[2] = wrap(psi + te - tp);
  out[3] = vp2;
  out[4] = ve2;
}

typedef struct {
  double dx, dphi, dvp, dve;
  size_t sy, sp, se, sv, n;
} sl_geom;

static sl_geom geom(const po_sl_cfg *c) {
  sl_geom g;
  const double pi = acos(-1.0);
  g.dx = 2 * c->extent / (c->nx - 1);
  g.dphi = 2 * pi / c->nh;
  g.dvp = (c->vp_hi - c->vp_lo) / (c->nvp - 1);
  g.dve = (c->ve_hi - c->ve_lo) / (c->nve - 1);
  g.sy = (size_t)c->nx;
  g.sp = g.sy * c->nx;
  g.se = g.sp * c->nh;
  g.sv = g.se * c->nve;
  g.n = g.sv * c->nvp;
  return g;
}

/* Lower node and weight along one axis: clamped node, linear extrapolation
 * beyond a non-periodic end; psi periodic. */
static void locate(double f, int n, int periodic, int *j, double *w) {
  if (periodic) {
    double fl = floor(f);
    *w = f - fl;
    int k = (int)fmod(fl, (double)n);
    if (k < 0) k += n;
    *j = k;
    return;
  }
  int k = (int)floor(f);
  if (k < 0) k = 0;
  if (k > n - 2) k = n - 2;
  *j = k;
  *w = f - k;
}

double po_sl_interpolate(const po_sl_cfg *c, const double *V, const double s[5]) {
  const sl_geom g = geom(c);
  const double pi = acos(-1.0);
  int jv, je, jp, jy, jx;
  double wv, we, wp, wy, wx;
  locate((s[3] - c->vp_lo) / g.dvp, c->nvp, 0, &jv, &wv);
  locate((s[4] - c->ve_lo) / g.dve, c->nve, 0, &je, &we);
  locate((s[2] + pi) / g.dphi, c->nh, 1, &jp, &wp);
  locate((s[1] + c->extent) / g.dx, c->nx, 0, &jy, &wy);
  locate((s[0] + c->extent) / g.dx, c->nx, 0, &jx, &wx);
  const int jp1 = (jp + 1) % c->nh;
  double total = 0;
  for (int bv = 0; bv < 2; bv++)
    for (int be = 0; be < 2; be++)
      for (int bp = 0; bp < 2; bp++)
        for (int by = 0; by < 2; by++)
          for (int bx = 0; bx < 2; bx++) {
            const double w = (bv ? wv : 1 - wv) * (be ? we : 1 - we) *
                             (bp ? wp : 1 - wp) * (by ? wy : 1 - wy) *
                             (bx ? wx : 1 - wx);
            const size_t idx = (size_t)(jv + bv) * g.sv + (size_t)(je + be) * g.se +
                               (size_t)(bp ? jp1 : jp) * g.sp +
                               (size_t)(jy + by) * g.sy + (size_t)(jx + bx);
            total += w * V[idx];
          }
  return total;
}

/* Neutral-first evader preference (map_game_policy.py:12-18) as catalogue
 * indices 3*ia+ik: (0,0) (-a,0) (a,0) (0,-k) (0,k) (-a,-k) (-a,k) (a,-k) (a,k). */
static const int E_ORDER[9] = {4, 1, 7, 3, 5, 0, 2, 6, 8};

/* Backup of one cell (flat index j): new value and the chosen actions. */
static double backup_cell(const po_sl_cfg *c, const sl_geom *g, const double *V,
                          size_t j, int *pick_p, int *pick_e) {
  const double pi = acos(-1.0);
  const double beta = exp(-c->dt);
  const int ix = (int)(j % c->nx);
  const size_t row = j / c->nx;
  const int iy = (int)(row % c->nx);
  const int ip = (int)((row / c->nx) % c->nh);
  const int ie = (int)((row / ((size_t)c->nx * c->nh)) % c->nve);
  const int iv = (int)(row / ((size_t)c->nx * c->nh * c->nve));
  const double x = -c->extent + ix * g->dx, y = -c->extent + iy * g->dx;
  const double psi = -pi + ip * g->dphi;
  const double vp = c->vp_lo + iv * g->dvp, ve = c->ve_lo + ie * g->dve;
  double worst[9];
  int worst_e[9];
  for (int up = 0; up < 9; up++) {
    double w_best = -INFINITY, vals[9];
    int w_idx = E_ORDER[0];
    for (int ue = 0; ue < 9; ue++) {
      double s[5];
      po_sl_successor(c, x, y, psi, vp, ve, up, ue, s);
      double v = po_sl_interpolate(c, V, s);
      if (c->mode == PO_SL_MINTIME) v = v < 0 ? 0 : (v > 1 ? 1 : v);
      vals[ue] = v;
      if (v > w_best) w_best = v;
    }
    for (int r = 0; r < 9; r++)
      if (vals[E_ORDER[r]] >= w_best - 1e-7) {
        w_idx = E_ORDER[r];
        break;
      }
    worst[up] = w_best;
    worst_e[up] = w_idx;
  }
  double best = INFINITY;
  for (int up = 0; up < 9; up++)
    if (worst[up] < best) best = worst[up];
  /* pursuer tie rule: smallest (|k|, |a|, index) among near-minima */
  int pick = -1, pick_key = 1 << 30;
  for (int up = 0; up < 9; up++) {
    if (worst[up] > best + 1e-7) continue;
    const int ka = abs(up % 3 - 1), aa = abs(up / 3 - 1);
    const int key = (ka * 2 + aa) * 16 + up;
    if (key < pick_key) {
      pick_key = key;
      pick = up;
    }
  }
  if (pick_p) *pick_p = pick;
  if (pick_e) *pick_e = worst_e[pick];
  if (c->mode == PO_SL_TUBE) return best < V[j] ? best : V[j];
  const double d = hypot(x, y) - c->radius;
  return d <= 0 ? 0.0 : (1 - beta) + beta * best;
}

int po_sl_backup(const po_sl_cfg *c, const double *V, double *out,
                 uint8_t *policy_p, uint8_t *policy_e) {
  const sl_geom g = geom(c);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : bad)
  for (size_t j = 0; j < g.n; j++) {
    int pp, pe;
    const double value = backup_cell(c, &g, V, j, &pp, &pe);
    if (!isfinite(value)) bad = 1;
    out[j] = value;
    if (policy_p) policy_p[j] = (uint8_t)pp;
    if (policy_e) policy_e[j] = (uint8_t)pe;
  }
  return bad ? PO_ENONFINITE : 0;
}

void po_sl_backup_cells(const po_sl_cfg *c, const double *V, size_t count,
                        const int64_t *cells, double *out, uint8_t *policy_p,
                        uint8_t *policy_e) {
  const sl_geom g = geom(c);
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t i = 0; i < count; i++) {
    int pp, pe;
    out[i] = backup_cell(c, &g, V, (size_t)cells[i], &pp, &pe);
    if (policy_p) policy_p[i] = (uint8_t)pp;
    if (policy_e) policy_e[i] = (uint8_t)pe;
  }
}

/* Initial fields: TUBE: hypot(x, y) - radius; MINTIME: 0 inside the capture
 * disk, 1 elsewhere (the cold start u = 1 - exp(-inf)). */
void po_sl_init(const po_sl_cfg *c, double *V) {
  const sl_geom g = geom(c);
  for (size_t row = 0; row < g.n / c->nx; row++) {
    const double y = -c->extent + (double)(row % c->nx) * g.dx;
    for (int ix = 0; ix < c->nx; ix++) {
      const double d = hypot(-c->extent + ix * g.dx, y) - c->radius;
      V[row * c->nx + ix] = c->mode == PO_SL_TUBE ? d : (d <= 0 ? 0.0 : 1.0);
    }
  }
}
