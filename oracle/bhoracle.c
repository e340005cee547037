/*
 * bhoracle.c -- CPU oracle (FP64) for the GRRT hot loop.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and the timed
 * CPU baseline.  Nothing in the product path links or calls this file.
 *
 * The arithmetic follows the reference operation by operation (same operand
 * order, no FMA contraction: build with -ffp-contract=off) so that the plugin
 * micro-kernels reproduce the reference's float64 results bit for bit.  Each
 * function cites the reference file:line it restates.
 */
#include "bhoracle.h"

#include <math.h>
#include <stddef.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NCOEF 11
static const double TWO_PI = 2.0 * 3.14159265358979323846;
static const double EPS_THETA = 1.0e-7; /* kerr.py:27 */

/* ------------------------------------------------------------------------- */
/* plugin micro-kernels                                                      */
/* ------------------------------------------------------------------------- */

/* lib.rs:61-73: first index whose grid value is > x (numpy searchsorted right). */
int64_t bho_search_right(const double *grid, int64_t n, double x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (x < grid[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

/* lib.rs:75-87, native_kernels.py:137-146 */
int bho_bracket_linear(const double *grid, int64_t n, double x, int64_t *i0, int64_t *i1, double *w) {
    if (x < grid[0] || x > grid[n - 1]) return 0;
    if (x == grid[n - 1]) {
        *i0 = n - 2;
        *i1 = n - 1;
        *w = 1.0;
        return 1;
    }
    int64_t right = bho_search_right(grid, n, x);
    int64_t lo = right - 1;
    if (lo < 0) lo = 0;
    if (lo > n - 2) lo = n - 2;
    *i0 = lo;
    *i1 = lo + 1;
    double den = grid[lo + 1] - grid[lo];
    if (den < 1.0e-300) den = 1.0e-300;
    *w = (x - grid[lo]) / den;
    return 1;
}

/* native_kernels.py:133-134 (Python float %), lib.rs:89-91 (rem_euclid). */
static double wrap_phi(double phi, double base) {
    double m = fmod(phi - base, TWO_PI);
    if (m < 0.0) m += TWO_PI;
    return m + base;
}

/* lib.rs:93-106, native_kernels.py:149-161 */
void bho_bracket_periodic_phi(const double *grid, int64_t n, double phi, int64_t *i0, int64_t *i1, double *w) {
    double p = wrap_phi(phi, grid[0]);
    int64_t lo = bho_search_right(grid, n, p) - 1;
    if (lo < 0) lo = n - 1;
    if (lo >= n) lo = n - 1;
    int64_t hi_i = (lo + 1) % n;
    double hi = hi_i > lo ? grid[hi_i] : grid[0] + TWO_PI;
    double pp = p >= grid[lo] ? p : p + TWO_PI;
    double den = hi - grid[lo];
    if (den < 1.0e-300) den = 1.0e-300;
    *i0 = lo;
    *i1 = hi_i;
    *w = (pp - grid[lo]) / den;
}

/* lib.rs:171-208, native_kernels.py:164-186 */
int bho_sample_one(const double *coeffs, const double *rg, int64_t nr, const double *tg, int64_t nt,
                   const double *pg, int64_t np, double r, double th, double ph, double out[11]) {
    int64_t r0, r1, t0, t1, p0, p1;
    double wr, wt, wp;
    if (!bho_bracket_linear(rg, nr, r, &r0, &r1, &wr) || !bho_bracket_linear(tg, nt, th, &t0, &t1, &wt)) {
        for (int c = 0; c < NCOEF; ++c) out[c] = NAN;
        return 0;
    }
    bho_bracket_periodic_phi(pg, np, ph, &p0, &p1, &wp);
#define OFF(ir, it, ip) ((((ir) * nt + (it)) * np + (ip)) * NCOEF)
    const double *c000 = coeffs + OFF(r0, t0, p0), *c001 = coeffs + OFF(r0, t0, p1);
    const double *c010 = coeffs + OFF(r0, t1, p0), *c011 = coeffs + OFF(r0, t1, p1);
    const double *c100 = coeffs + OFF(r1, t0, p0), *c101 = coeffs + OFF(r1, t0, p1);
    const double *c110 = coeffs + OFF(r1, t1, p0), *c111 = coeffs + OFF(r1, t1, p1);
#undef OFF
    double owp = 1.0 - wp, owt = 1.0 - wt, owr = 1.0 - wr;
    for (int c = 0; c < NCOEF; ++c) {
        double c00 = owp * c000[c] + wp * c001[c];
        double c01 = owp * c010[c] + wp * c011[c];
        double c10 = owp * c100[c] + wp * c101[c];
        double c11 = owp * c110[c] + wp * c111[c];
        double cc0 = owt * c00 + wt * c01;
        double cc1 = owt * c10 + wt * c11;
        out[c] = owr * cc0 + wr * cc1;
    }
    return 1;
}

/* lib.rs:37-59, native_kernels.py:213-222: dS/ds = j - K S with
 * K = [[aI,aQ,aU,aV],[aQ,aI,rV,-rU],[aU,-rV,aI,rQ],[aV,rU,-rQ,aI]]. */
void bho_stokes_rhs(const double s[4], const double c[11], double out[4]) {
    out[0] = c[0] - (c[4] * s[0] + c[5] * s[1] + c[6] * s[2] + c[7] * s[3]);
    out[1] = c[1] - (c[5] * s[0] + c[4] * s[1] + c[8] * s[2] - c[10] * s[3]);
    out[2] = c[2] - (c[6] * s[0] - c[8] * s[1] + c[4] * s[2] + c[9] * s[3]);
    out[3] = c[3] - (c[7] * s[0] + c[10] * s[1] - c[9] * s[2] + c[4] * s[3]);
}

/* lib.rs:210-225 */
void bho_stokes_step_rk2(double s[4], const double c[11], double ds) {
    double k1[4], mid[4], k2[4];
    double hds = 0.5 * ds;
    bho_stokes_rhs(s, c, k1);
    for (int i = 0; i < 4; ++i) mid[i] = s[i] + hds * k1[i];
    bho_stokes_rhs(mid, c, k2);
    for (int i = 0; i < 4; ++i) s[i] = s[i] + ds * k2[i];
}

/* lib.rs:227-279 */
void bho_stokes_rk2_brick(const double *coeffs, int64_t cells, double ds, const double *initial,
                          int64_t initial_len, double *out) {
    int broadcast = initial_len == 4;
    for (int64_t i = 0; i < cells; ++i) {
        const double *s0 = initial + (broadcast ? 0 : 4 * i);
        double s[4] = {s0[0], s0[1], s0[2], s0[3]};
        bho_stokes_step_rk2(s, coeffs + NCOEF * i, ds);
        memcpy(out + 4 * i, s, sizeof s);
    }
}

/* lib.rs:281-306 */
void bho_sample_brick_trilinear(const double *coeffs, const double *rg, int64_t nr, const double *tg,
                                int64_t nt, const double *pg, int64_t np, const double *points,
                                int64_t n, double *out) {
    for (int64_t i = 0; i < n; ++i)
        bho_sample_one(coeffs, rg, nr, tg, nt, pg, np, points[3 * i], points[3 * i + 1], points[3 * i + 2],
                       out + NCOEF * i);
}

/* lib.rs:308-366 (NaN rows), then native_kernels.py:342-350 (policy). */
void bho_sample_and_step_stokes(const double *coeffs, const double *rg, int64_t nr, const double *tg,
                                int64_t nt, const double *pg, int64_t np, const double *points,
                                int64_t n, double ds, const double *initial, int64_t initial_len,
                                int policy, double *out) {
    int broadcast = initial_len == 4;
    for (int64_t i = 0; i < n; ++i) {
        double c[NCOEF];
        const double *s0 = initial + (broadcast ? 0 : 4 * i);
        double *o = out + 4 * i;
        if (!bho_sample_one(coeffs, rg, nr, tg, nt, pg, np, points[3 * i], points[3 * i + 1], points[3 * i + 2],
                            c)) {
            for (int k = 0; k < 4; ++k) o[k] = policy == 1 ? s0[k] : (policy == 2 ? 0.0 : NAN);
            continue;
        }
        double s[4] = {s0[0], s0[1], s0[2], s0[3]};
        bho_stokes_step_rk2(s, c, ds);
        memcpy(o, s, sizeof s);
    }
}

/* native_kernels.py:189-210 (inclusive bounds, phi ignored) */
void bho_sample_brick_valid_mask(const double *rg, int64_t nr, const double *tg, int64_t nt,
                                 const double *points, int64_t n, uint8_t *mask) {
    for (int64_t i = 0; i < n; ++i) {
        double r = points[3 * i], th = points[3 * i + 1];
        mask[i] = (uint8_t)((r >= rg[0]) & (r <= rg[nr - 1]) & (th >= tg[0]) & (th <= tg[nt - 1]));
    }
}

/* ------------------------------------------------------------------------- */
/* Kerr geometry                                                             */
/* ------------------------------------------------------------------------- */

/* kerr.py:35-36 */
double bho_safe_theta(double th) {
    double lo = EPS_THETA, hi = 3.14159265358979323846 - EPS_THETA;
    if (th < lo) return lo;   /* np.clip keeps NaN */
    if (th > hi) return hi;
    return th;
}

/* kerr.py:39-42 */
double bho_horizon_radius(double a) { return 1.0 + sqrt(1.0 - a * a); }

/* kerr.py:52-64 */
static double k_sigma(double r, double th, double a) { return r * r + a * a * pow(cos(th), 2.0); }
static double k_delta(double r, double a) { return r * r - 2.0 * r + a * a; }
static double k_big_a(double r, double th, double a) {
    double s2 = pow(sin(th), 2.0);
    return pow(r * r + a * a, 2.0) - a * a * k_delta(r, a) * s2;
}

/* kerr.py:67-83 */
void bho_metric_cov(double r, double theta, double a, double g[16]) {
    double th = bho_safe_theta(theta);
    double sig = k_sigma(r, th, a), dlt = k_delta(r, a);
    double s = sin(th), s2 = s * s, A = k_big_a(r, th, a);
    memset(g, 0, 16 * sizeof(double));
    g[0] = -(1.0 - 2.0 * r / sig);
    g[3] = g[12] = -2.0 * a * r * s2 / sig;
    g[5] = sig / dlt;
    g[10] = sig;
    g[15] = A * s2 / sig;
}

/* kerr.py:86-102 */
void bho_metric_con(double r, double theta, double a, double g[16]) {
    double th = bho_safe_theta(theta);
    double sig = k_sigma(r, th, a), dlt = k_delta(r, a);
    double s = sin(th), s2 = s * s, A = k_big_a(r, th, a);
    if (s2 < EPS_THETA * EPS_THETA) s2 = EPS_THETA * EPS_THETA;
    memset(g, 0, 16 * sizeof(double));
    g[0] = -A / (sig * dlt);
    g[3] = g[12] = -2.0 * a * r / (sig * dlt);
    g[5] = dlt / sig;
    g[10] = 1.0 / sig;
    g[15] = (dlt - a * a * s2) / (sig * dlt * s2);
}

/* kerr.py:236-282: analytic d g^{mu nu} / dr (wrt_theta = 0) or / dtheta. */
void bho_metric_derivative(double r, double theta, double a, int wrt_theta, double out[16]) {
    double th = bho_safe_theta(theta);
    double s = sin(th), c = cos(th);
    double s2 = s * s;
    if (s2 < EPS_THETA * EPS_THETA) s2 = EPS_THETA * EPS_THETA;
    double ds2 = 2.0 * s * c;
    double sig = k_sigma(r, th, a), dlt = k_delta(r, a), A = k_big_a(r, th, a);
    double sig_p, dlt_p, A_p, s2_p;
    if (!wrt_theta) {
        sig_p = 2.0 * r;
        dlt_p = 2.0 * r - 2.0;
        A_p = 4.0 * r * (r * r + a * a) - a * a * dlt_p * s2;
        s2_p = 0.0;
    } else {
        sig_p = -a * a * ds2;
        dlt_p = 0.0;
        A_p = -a * a * dlt * ds2;
        s2_p = ds2;
    }
    memset(out, 0, 16 * sizeof(double));
    double den = sig * dlt;
    double den_p = sig_p * dlt + sig * dlt_p;
    out[0] = -((A_p * den - A * den_p) / (den * den));
    double num = -2.0 * a * r;
    double num_p = !wrt_theta ? -2.0 * a : 0.0;
    out[3] = out[12] = (num_p * den - num * den_p) / (den * den);
    out[5] = (dlt_p * sig - dlt * sig_p) / (sig * sig);
    out[10] = -sig_p / (sig * sig);
    num = dlt - a * a * s2;
    num_p = dlt_p - a * a * s2_p;
    den = sig * dlt * s2;
    den_p = sig_p * dlt * s2 + sig * dlt_p * s2 + sig * dlt * s2_p;
    out[15] = (num_p * den - num * den_p) / (den * den);
}

/* p @ M @ p for a 4x4 row-major matrix (left to right, as numpy's matmul chain). */
static double quad(const double p[4], const double m[16]) {
    double v[4];
    for (int j = 0; j < 4; ++j) v[j] = p[0] * m[j] + p[1] * m[4 + j] + p[2] * m[8 + j] + p[3] * m[12 + j];
    return v[0] * p[0] + v[1] * p[1] + v[2] * p[2] + v[3] * p[3];
}

/* kerr.py:113-121: H = 0.5 * pcov @ gcon @ pcov, evaluated as ((0.5 p) @ g) @ p */
double bho_hamiltonian(const double y[6], double a, double pt, double pphi) {
    double p[4] = {pt, y[4], y[5], pphi}, g[16];
    bho_metric_con(y[1], y[2], a, g);
    double hp[4] = {0.5 * p[0], 0.5 * p[1], 0.5 * p[2], 0.5 * p[3]};
    double v[4];
    for (int j = 0; j < 4; ++j) v[j] = hp[0] * g[j] + hp[1] * g[4 + j] + hp[2] * g[8 + j] + hp[3] * g[12 + j];
    return v[0] * p[0] + v[1] * p[1] + v[2] * p[2] + v[3] * p[3];
}

/* kerr.py:285-303 */
void bho_geodesic_rhs(const double y[6], double a, double pt, double pphi, double dy[6]) {
    double r = y[1], th = bho_safe_theta(y[2]);
    double p[4] = {pt, y[4], y[5], pphi}, g[16], dr[16], dth[16];
    bho_metric_con(r, th, a, g);
    for (int i = 0; i < 4; ++i) dy[i] = g[4 * i] * p[0] + g[4 * i + 1] * p[1] + g[4 * i + 2] * p[2] + g[4 * i + 3] * p[3];
    bho_metric_derivative(r, th, a, 0, dr);
    bho_metric_derivative(r, th, a, 1, dth);
    dy[4] = -0.5 * quad(p, dr);
    dy[5] = -0.5 * quad(p, dth);
}

/* RK2 midpoint step: native/cuda/kerr_stokes_kernel.cu:13 form
 * (k1; mid = y + h/2 k1; k2 = f(mid); y + h k2), theta clamped as kerr.py:312. */
void bho_rk2_step(const double y[6], double h, double a, double pt, double pphi, double out[6]) {
    double k1[6], mid[6], k2[6];
    double hh = 0.5 * h;
    bho_geodesic_rhs(y, a, pt, pphi, k1);
    for (int i = 0; i < 6; ++i) mid[i] = y[i] + hh * k1[i];
    bho_geodesic_rhs(mid, a, pt, pphi, k2);
    for (int i = 0; i < 6; ++i) out[i] = y[i] + h * k2[i];
    out[2] = bho_safe_theta(out[2]);
}

static int all_finite6(const double y[6]);

/* kerr.py:306-313: classical RK4, theta clamped. */
void bho_rk4_step(const double y[6], double h, double a, double pt, double pphi, double out[6]) {
    double k1[6], k2[6], k3[6], k4[6], tmp[6];
    double hh = 0.5 * h;
    bho_geodesic_rhs(y, a, pt, pphi, k1);
    for (int i = 0; i < 6; ++i) tmp[i] = y[i] + hh * k1[i];
    bho_geodesic_rhs(tmp, a, pt, pphi, k2);
    for (int i = 0; i < 6; ++i) tmp[i] = y[i] + hh * k2[i];
    bho_geodesic_rhs(tmp, a, pt, pphi, k3);
    for (int i = 0; i < 6; ++i) tmp[i] = y[i] + h * k3[i];
    bho_geodesic_rhs(tmp, a, pt, pphi, k4);
    double h6 = h / 6.0;
    for (int i = 0; i < 6; ++i) out[i] = y[i] + h6 * (((k1[i] + 2.0 * k2[i]) + 2.0 * k3[i]) + k4[i]);
    out[2] = bho_safe_theta(out[2]);
}

/* kerr.py:337-384 trace_kerr_null_geodesic with store_stride 1: writes the
 * stored states (at most max_steps + 1 rows of 6) and returns their count;
 * *status: 0 max_steps, 1 captured, 2 escaped, 3 invalid. */
int64_t bho_trace_rk4(const double y0[6], double pt, double pphi, double a, double h, int32_t max_steps,
                      double escape_radius, double *states, int32_t *status) {
    double y[6], yn[6];
    memcpy(y, y0, sizeof y);
    memcpy(states, y, sizeof y);
    int64_t n = 1;
    double r_capture = bho_horizon_radius(a) * (1.0 + 2.0e-4);
    double prev_r = y[1];
    *status = BHO_STATUS_MAX_STEPS;
    for (int32_t i = 1; i <= max_steps; ++i) {
        bho_rk4_step(y, h, a, pt, pphi, yn);
        if (!all_finite6(yn)) {
            *status = BHO_STATUS_INVALID;
            break;
        }
        memcpy(y, yn, sizeof y);
        memcpy(states + 6 * n, y, sizeof y);
        ++n;
        if (y[1] <= r_capture) {
            *status = BHO_STATUS_CAPTURED;
            break;
        }
        if (y[1] > escape_radius && y[1] > prev_r) {
            *status = BHO_STATUS_ESCAPED;
            break;
        }
        prev_r = y[1];
    }
    return n;
}

/* kerr.py:188-233 camera_ray_initial_state with kerr.py:124-152 zamo_tetrad. */
int bho_camera_ray(const bho_view *v, double ndc_x, double ndc_y, double aspect, double y0[6], double *pt,
                   double *pphi) {
    const double deg = 3.14159265358979323846 / 180.0; /* math.radians */
    double a = v->spin_a;
    double th = bho_safe_theta(v->theta_obs);
    double fov_y = v->fov_y_deg * deg;
    double tan_y = tan(0.5 * fov_y);
    double tan_x = aspect * tan_y;
    double n[3] = {-1.0, -ndc_y * tan_y, ndc_x * tan_x};
    if (v->roll_deg != 0.0) {
        double roll = v->roll_deg * deg, ct = cos(roll), st = sin(roll);
        double nt = ct * n[1] - st * n[2], np_ = st * n[1] + ct * n[2];
        n[1] = nt;
        n[2] = np_;
    }
    double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int i = 0; i < 3; ++i) n[i] = n[i] / nn;

    double r = v->r_obs;
    double sig = k_sigma(r, th, a), dlt = k_delta(r, a), A = k_big_a(r, th, a);
    if (dlt <= 0.0) return -1;
    double s = sin(th);
    double gcov[16];
    bho_metric_cov(r, th, a, gcov);
    double lapse = sqrt(sig * dlt / A);
    double omega = 2.0 * a * r / A;
    if (fabs(s) < EPS_THETA) return -1;
    double tet[4][4] = {{1.0 / lapse, 0.0, 0.0, omega / lapse},
                        {0.0, sqrt(dlt / sig), 0.0, 0.0},
                        {0.0, 0.0, 1.0 / sqrt(sig), 0.0},
                        {0.0, 0.0, 0.0, 1.0 / sqrt(gcov[15])}};
    double pcon[4], pcov[4];
    for (int i = 0; i < 4; ++i) pcon[i] = tet[0][i] + n[0] * tet[1][i] + n[1] * tet[2][i] + n[2] * tet[3][i];
    for (int i = 0; i < 4; ++i)
        pcov[i] = gcov[4 * i] * pcon[0] + gcov[4 * i + 1] * pcon[1] + gcov[4 * i + 2] * pcon[2] + gcov[4 * i + 3] * pcon[3];
    y0[0] = 0.0;
    y0[1] = r;
    y0[2] = th;
    y0[3] = v->phi_obs;
    y0[4] = pcov[1];
    y0[5] = pcov[2];
    *pt = pcov[0];
    *pphi = pcov[3];
    return 0;
}

static int all_finite6(const double y[6]) {
    for (int i = 0; i < 6; ++i)
        if (!isfinite(y[i])) return 0;
    return 1;
}

/* One pixel: accelerated_renderer.py:136-143 pixel setup, kerr.py:337-384
 * trace (RK2, h = clamp(h_scale * r, h_min, h_max)), and the streaming form of
 * accelerated_renderer.py:100-126 (each stored segment is consumed as soon as
 * it is produced; the arithmetic per segment is unchanged). */
void bho_trace_pixel(const bho_view *v, const double *coeffs, const double *rg, int64_t nr, const double *tg,
                     int64_t nt, const double *pg, int64_t np, int32_t px, int32_t py, int stop_at_tau,
                     bho_ray_result *res) {
    double aspect = (double)v->width / (double)v->height;
    double ndc_y = 1.0 - 2.0 * ((double)py + 0.5) / (double)v->height;
    double ndc_x = 2.0 * ((double)px + 0.5) / (double)v->width - 1.0;
    double y[6], pt, pphi;
    memset(res, 0, sizeof *res);
    res->status = BHO_STATUS_INVALID;
    if (bho_camera_ray(v, ndc_x, ndc_y, aspect, y, &pt, &pphi) != 0) return;

    double a = v->spin_a;
    double r_plus = bho_horizon_radius(a);
    double r_capture = r_plus * (1.0 + 2.0e-4);
    double H0 = fabs(bho_hamiltonian(y, a, pt, pphi));
    double max_h_err = 0.0;
    double prev_r = y[1];
    double S[4] = {0.0, 0.0, 0.0, 0.0};
    double tau = 0.0;
    int transfer_done = 0;
    int status = BHO_STATUS_MAX_STEPS;
    int32_t steps = 0, in_brick = 0;
    /* Optional horizon guard (not part of the reference): an inbound ray inside
     * both the innermost spherical photon orbit (prograde equatorial circular
     * orbit, r = 2(1 + cos(2/3 acos(-|a|)))) and the brick's inner radius can
     * add no more emission in exact arithmetic, so it is captured there.  A
     * step whose RK2 midpoint (the Euler half step) lies inside the horizon is
     * not taken either: its second stage would be evaluated where Delta < 0,
     * which flings the ray back out with garbage momenta; the ray is captured
     * at that step's start. */
    const double r_guard = (v->flags & 1) ? fmin(2.0 * (1.0 + cos((2.0 / 3.0) * acos(-fabs(a)))), rg[0]) : 0.0;
    for (int i = 1; i <= v->max_steps; ++i) {
        if (y[1] < r_guard && y[4] < 0.0) {
            status = BHO_STATUS_CAPTURED;
            break;
        }
        double h = v->h_scale * y[1];
        if (h < v->h_min) h = v->h_min;
        if (h > v->h_max) h = v->h_max;
        if (r_guard > 0.0) {
            double k1[6];
            bho_geodesic_rhs(y, a, pt, pphi, k1);
            if (y[1] + 0.5 * h * k1[1] < r_plus) {
                status = BHO_STATUS_CAPTURED;
                break;
            }
        }
        double yn[6];
        bho_rk2_step(y, h, a, pt, pphi, yn);
        steps++;
        int finite = all_finite6(yn);
        if (finite) {
            double H = fabs(bho_hamiltonian(yn, a, pt, pphi));
            double e = fabs(H - H0);
            if (e > max_h_err) max_h_err = e;
        }
        /* segment (y, yn): accelerated_renderer.py:113-125 */
        if (!transfer_done) {
            double mid[3] = {0.5 * (y[1] + yn[1]), 0.5 * (y[2] + yn[2]), 0.5 * (y[3] + yn[3])};
            double c[NCOEF];
            if (bho_sample_one(coeffs, rg, nr, tg, nt, pg, np, mid[0], mid[1], mid[2], c)) {
                in_brick++;
                double d0 = yn[1] - y[1], d1 = yn[2] - y[2], d2 = yn[3] - y[3];
                double dl = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                if (1.0e-14 > dl) dl = 1.0e-14; /* Python max(dlambda, 1e-14): NaN propagates */
                double ds = v->affine_to_length_cm * dl;
                if (ds < 0.0) ds = 0.0;
                bho_stokes_step_rk2(S, c, ds);
                double ai = 0.0 > c[4] ? 0.0 : c[4]; /* Python max(alpha_i, 0.0) */
                tau += ai * ds;
                if (tau >= v->max_optical_depth) transfer_done = 1;
            }
        }
        memcpy(y, yn, sizeof y);
        if (!finite) {
            status = BHO_STATUS_INVALID;
            break;
        }
        if (transfer_done && stop_at_tau) {
            status = 4; /* optically thick: the trace ends at the cutoff */
            break;
        }
        double r = y[1];
        if (r <= r_capture) {
            status = BHO_STATUS_CAPTURED;
            break;
        }
        if (r > v->escape_radius && r > prev_r) {
            status = BHO_STATUS_ESCAPED;
            break;
        }
        prev_r = r;
    }
    for (int k = 0; k < 4; ++k) res->stokes[k] = isfinite(S[k]) ? S[k] : 0.0; /* np.nan_to_num(nan=0, inf=0) */
    res->h_drift = max_h_err;
    res->tau = tau;
    res->steps = steps;
    res->in_brick = in_brick;
    res->status = status;
}

void bho_render(const bho_view *v, const double *coeffs, const double *rg, int64_t nr, const double *tg,
                int64_t nt, const double *pg, int64_t np, int stop_at_tau, int n_threads, double *out,
                int32_t *steps, int32_t *status, double *h_drift) {
    int64_t npix = (int64_t)v->crop_w * v->crop_h;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(n_threads)
#endif
    for (int64_t k = 0; k < npix; ++k) {
        int32_t px = v->x0 + (int32_t)(k % v->crop_w);
        int32_t py = v->y0 + (int32_t)(k / v->crop_w);
        bho_ray_result res;
        bho_trace_pixel(v, coeffs, rg, nr, tg, nt, pg, np, px, py, stop_at_tau, &res);
        memcpy(out + 4 * k, res.stokes, sizeof res.stokes);
        if (steps) steps[k] = res.steps;
        if (status) status[k] = res.status;
        if (h_drift) h_drift[k] = res.h_drift;
    }
    (void)n_threads;
}

int bho_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
