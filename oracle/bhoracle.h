/*
 * bhoracle.h -- CPU oracle (FP64) for the GRRT hot loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm used as the parity checker for the CUDA path and as the timed CPU
 * baseline.  Only tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load it; the product path never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the reference project root).
 */
#ifndef BHORACLE_H
#define BHORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- plugin micro-kernels (native/core/src/lib.rs, python/blackhole_sim/native_kernels.py) ---- */

/* lib.rs:61-73 search_right == numpy.searchsorted(side="right"). */
int64_t bho_search_right(const double *grid, int64_t n, double x);

/* lib.rs:75-87, native_kernels.py:137-146.  Returns 1 and (i0, i1, w) when x is
 * inside [grid[0], grid[n-1]] (NaN passes, as in the reference), else 0. */
int bho_bracket_linear(const double *grid, int64_t n, double x, int64_t *i0, int64_t *i1, double *w);

/* lib.rs:89-106, native_kernels.py:133-161. */
void bho_bracket_periodic_phi(const double *grid, int64_t n, double phi, int64_t *i0, int64_t *i1, double *w);

/* lib.rs:171-208, native_kernels.py:164-186.  Returns 1 when valid (out filled),
 * 0 when outside the nonperiodic r/theta domain (out filled with NaN). */
int bho_sample_one(const double *coeffs, const double *rg, int64_t nr, const double *tg, int64_t nt,
                   const double *pg, int64_t np, double r, double th, double ph, double out[11]);

/* lib.rs:37-59, native_kernels.py:213-222. */
void bho_stokes_rhs(const double s[4], const double c[11], double out[4]);

/* lib.rs:210-225, native_kernels.py:279-293. */
void bho_stokes_step_rk2(double s[4], const double c[11], double ds);

/* lib.rs:227-279 (native returns flat list). initial_len is 4 or 4*cells. */
void bho_stokes_rk2_brick(const double *coeffs, int64_t cells, double ds, const double *initial,
                          int64_t initial_len, double *out);

/* lib.rs:281-306. out has n*11 values; NaN rows for out-of-domain samples. */
void bho_sample_brick_trilinear(const double *coeffs, const double *rg, int64_t nr, const double *tg,
                                int64_t nt, const double *pg, int64_t np, const double *points,
                                int64_t n, double *out);

/* lib.rs:308-366 plus the invalid_policy post-processing of
 * native_kernels.py:325-351 (policy 0 = "nan", 1 = "initial", 2 = "zero"). */
void bho_sample_and_step_stokes(const double *coeffs, const double *rg, int64_t nr, const double *tg,
                                int64_t nt, const double *pg, int64_t np, const double *points,
                                int64_t n, double ds, const double *initial, int64_t initial_len,
                                int policy, double *out);

/* native_kernels.py:189-210. */
void bho_sample_brick_valid_mask(const double *rg, int64_t nr, const double *tg, int64_t nt,
                                 const double *points, int64_t n, uint8_t *mask);

/* ---- Kerr geometry (python/blackhole_sim/kerr.py) ---- */

double bho_safe_theta(double th);                                         /* kerr.py:35-36 */
double bho_horizon_radius(double a);                                      /* kerr.py:39-42 */
void bho_metric_cov(double r, double th, double a, double g[16]);         /* kerr.py:67-83 */
void bho_metric_con(double r, double th, double a, double g[16]);         /* kerr.py:86-102 */
void bho_metric_derivative(double r, double th, double a, int wrt_theta, double out[16]); /* kerr.py:236-282 */
double bho_hamiltonian(const double y[6], double a, double pt, double pphi); /* kerr.py:113-121 */
void bho_geodesic_rhs(const double y[6], double a, double pt, double pphi, double dy[6]); /* kerr.py:285-303 */
/* RK2 midpoint step (native/cuda/kerr_stokes_kernel.cu:13 form) on the analytic
 * RHS, theta clamped like kerr.py:312. */
void bho_rk2_step(const double y[6], double h, double a, double pt, double pphi, double out[6]);
void bho_rk4_step(const double y[6], double h, double a, double pt, double pphi, double out[6]);
int64_t bho_trace_rk4(const double y0[6], double pt, double pphi, double a, double h, int32_t max_steps,
                      double escape_radius, double *states, int32_t *status);

/* One camera view: kerr.py:155-233 LocalCamera + accelerated_renderer.py:36-46. */
typedef struct bho_view {
    double spin_a;
    double r_obs, theta_obs, phi_obs;     /* radians for angles */
    double fov_y_deg, roll_deg;
    double h_scale, h_min, h_max;         /* h = clamp(h_scale * r, h_min, h_max) */
    double escape_radius;
    double affine_to_length_cm;           /* the "or 1.0" of accelerated_renderer.py:146 applied by caller */
    double max_optical_depth;
    int32_t width, height;                /* full image (NDC) */
    int32_t x0, y0, crop_w, crop_h;       /* rendered rectangle */
    int32_t max_steps;
    int32_t flags;                        /* bit 0: horizon guard (not in the reference; see bhoracle.c) */
} bho_view;

enum { BHO_STATUS_MAX_STEPS = 0, BHO_STATUS_CAPTURED = 1, BHO_STATUS_ESCAPED = 2, BHO_STATUS_INVALID = 3 };

/* kerr.py:188-233.  Returns 0 on success, -1 when the ZAMO tetrad is undefined. */
int bho_camera_ray(const bho_view *v, double ndc_x, double ndc_y, double aspect, double y0[6], double *pt,
                   double *pphi);

typedef struct bho_ray_result {
    double stokes[4];
    double h_drift;      /* max |H - H0| over executed steps (kerr.py:352,367) */
    double tau;          /* optical depth accumulated (accelerated_renderer.py:123) */
    int32_t steps;       /* geodesic steps executed */
    int32_t in_brick;    /* steps whose midpoint sample was valid */
    int32_t status;      /* BHO_STATUS_* */
    int32_t pad;
} bho_ray_result;

/* One pixel of the brick renderer: camera -> RK2 trace with kerr.py:337-384
 * termination -> accelerated_renderer.py:100-126 accumulation.  The brick is
 * float64 [nr][nt][np][11] in COEFF_NAMES order.  When stop_at_tau is nonzero
 * the trace ends at the optical-depth cutoff (the geodesic steps after that
 * point cannot change the Stokes vector). */
void bho_trace_pixel(const bho_view *v, const double *coeffs, const double *rg, int64_t nr, const double *tg,
                     int64_t nt, const double *pg, int64_t np, int32_t px, int32_t py, int stop_at_tau,
                     bho_ray_result *res);

/* Render the crop rectangle of a view; out is crop_h*crop_w*4 doubles (row-major),
 * steps/status/h_drift may be NULL.  n_threads <= 0 uses all OpenMP threads. */
void bho_render(const bho_view *v, const double *coeffs, const double *rg, int64_t nr, const double *tg,
                int64_t nt, const double *pg, int64_t np, int stop_at_tau, int n_threads, double *out,
                int32_t *steps, int32_t *status, double *h_drift);

/* Threads the OpenMP runtime would use. */
int bho_max_threads(void);

#ifdef __cplusplus
}
#endif

#endif
