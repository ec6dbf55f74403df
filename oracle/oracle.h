/*
 * CPU ORACLE — test infrastructure only (see relative5d.c).  These functions
 * are the checker for the CUDA path: tests, the smoke check and the CPU
 * baseline leg of bench.py call them; the product never does.
 */
#ifndef PE_ORACLE_H
#define PE_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#define PO_ENOMEM (-2)
#define PO_ENONFINITE (-3)
#define PO_EINVAL (-1)

/* Relative 5D game: storage [vP, vE, psi, y, x], x fastest. */
typedef struct {
  int nx, nh, nvp, nve, order;
  double extent, radius, vp_lo, vp_hi, ve_lo, ve_hi, acc_p, acc_e, curv_p,
      curv_e, cfl;
} po_rel_cfg;

size_t po_rel_cells(const po_rel_cfg *c);
double po_rel_cfl_limit(const po_rel_cfg *c);
void po_rel_init(const po_rel_cfg *c, float *field, float *arrival);
void po_rel_init_f64(const po_rel_cfg *c, double *field);
int po_rel_stage_f32(const po_rel_cfg *c, const float *src, float *dst,
                     float *arrival, double dt, double t, int blend,
                     double *max_increase);
int po_rel_stage_f64(const po_rel_cfg *c, const double *src, double *dst,
                     double dt, int blend);
int po_rel_solve_f32(const po_rel_cfg *c, double horizon, double output_dt,
                     float *frames, float *arrival, long *steps_out);
int po_rel_solve_f64(const po_rel_cfg *c, double horizon, double output_dt,
                     double *final, long *steps_out);

/* Legacy 6D square game: storage [xP, yP, thP, xE, yE, thE], thE fastest;
 * constant speeds vp, ve and turn-rate bounds wp, we. */
typedef struct {
  int n, nh, order;
  float extent, arena, radius, vp, ve, wp, we;
  double cfl;
} po_s6_cfg;

size_t po_s6_cells(const po_s6_cfg *c);
double po_s6_dt_limit(const po_s6_cfg *c);
/* max(target, avoid) and arrival = 0 where <= 0, NaN elsewhere. */
void po_s6_init(const po_s6_cfg *c, float *a, float *arrival);
/* One stage; base != NULL: the RK2 average, tube minimum and avoid floor. */
int po_s6_stage(const po_s6_cfg *c, const float *src, float *dst, const float *base,
                float *arrival, float dt, double tau);

/* Dense 8D game: storage [xP, yP, thP, vP, xE, yE, thE, vE], vE fastest. */
typedef struct {
  int n, nh, np, ne, order;
  int linear_speed;  /* 1: inward one-sided slopes at the speed bounds */
  int avoid_square;  /* 1: reference square-arena avoid floor; 0: none */
  float extent, arena, radius, p_lo, p_hi, e_lo, e_hi, ap, ae, kp, ke;
  double cfl;
} po_w8_cfg;

size_t po_w8_cells(const po_w8_cfg *c);
double po_w8_dt_limit(const po_w8_cfg *c);
void po_w8_init_square(const po_w8_cfg *c, float *a, float *arrival);
double po_rect_separation(double px, double py, double pth, double ex,
                          double ey, double eth, double p_len, double p_wid,
                          double e_len, double e_wid);
void po_w8_init_contact(const po_w8_cfg *c, double p_len, double p_wid,
                        double e_len, double e_wid, float *a, float *arrival);
int po_w8_stage(const po_w8_cfg *c, const float *src, float *dst,
                const float *base, float *arrival, float dt, double tau);
/* Obstacle map game (clearances per (x, y, heading) pose of each car). */
void po_w8_init_map(const po_w8_cfg *c, const float *p_clear, const float *e_clear,
                    float *a, float *arrival);
int po_w8_stage_clear(const po_w8_cfg *c, const float *src, float *dst, const float *base,
                      float *arrival, float dt, double tau, const float *p_clear);
/* The same stage in double precision on double fields (no arrival): the
 * rounding-free reference for float32 variants of the step. */
int po_w8_stage_f64(const po_w8_cfg *c, const double *src, double *dst,
                    const double *base, double dt);

/* Relative 5D semi-Lagrangian backup (FP64). */
#define PO_SL_TUBE 0
#define PO_SL_MINTIME 1
typedef struct {
  int nx, nh, nvp, nve, mode;
  double extent, radius, vp_lo, vp_hi, ve_lo, ve_hi, acc_p, acc_e, curv_p,
      curv_e, dt;
} po_sl_cfg;

void po_sl_integrated_speed(double v, double a, double dt, double vmin,
                            double vmax, double *v_out, double *dist);
void po_sl_successor(const po_sl_cfg *c, double x, double y, double psi,
                     double vp, double ve, int up, int ue, double out[5]);
double po_sl_interpolate(const po_sl_cfg *c, const double *V, const double s[5]);
int po_sl_backup(const po_sl_cfg *c, const double *V, double *out,
                 uint8_t *policy_p, uint8_t *policy_e);
void po_sl_backup_cells(const po_sl_cfg *c, const double *V, size_t count,
                        const int64_t *cells, double *out, uint8_t *policy_p,
                        uint8_t *policy_e);
void po_sl_init(const po_sl_cfg *c, double *V);

/* Bits in which the exact stage's division by a spacing b (through RN(1/b)
 * and one FMA correction) differs from a / b, over n drawn dividends. */
long long po_div_const_check(double b, long long n, unsigned long long seed);
long long po_div_const_checkf(float b, long long n, unsigned long long seed);

#endif
