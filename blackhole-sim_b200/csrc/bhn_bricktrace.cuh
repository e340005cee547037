// bhn_bricktrace.cuh -- the reference's own brick renderer loop (FP64).
// Included at the end of bhn_render.cu (camera, metric RHS).
//
// python/blackhole_sim/accelerated_renderer.py:100-158: per pixel the camera
// ray (kerr.py:188-233), the fixed-step RK4 trace (kerr.py:306-313, 337-384),
// then integrate_stokes_from_bricks_trace over consecutive states: the brick
// sampled trilinearly at the segment midpoint (sample_coefficient_brick,
// :73-97: no sample outside the nonperiodic r / theta range),
// ds = L max(|d(r, theta, phi)|, 1e-14), one RK2 or exact Stokes step,
// tau += max(alpha_I, 0) ds until tau reaches the cutoff, and the final
// nan_to_num(nan = posinf = neginf = 0).  Unlike the fused renderer
// (bhn_render_launch: the RK2 step h = 0.02 r), this is the reference
// Python's method, one thread per ray.

#include "bhn_exact.cuh"
#include "bhn_transfer.cuh"

namespace bhn {

// Whether a ray at radius r, moving out (p_r > 0), keeps moving out for good.
// With E = -p_t, L = p_phi, the state's own 2H = g^{mu nu} p_mu p_nu (the
// fixed-step integrator's drift from the null value 0, up to ~1e-3 E^2 after
// a pass near the hole) and the Carter constant of that H,
// K = p_theta^2 + (L / sin - a E sin)^2 - 2H a^2 cos^2, the radial motion obeys
// (Delta p_r)^2 = R(r) = (E (r^2 + a^2) - a L)^2 - Delta (K - 2H r^2)
//                     = (E^2 + 2H) r^4 - 4H r^3 + c2 r^2 + 2K r + c0,
// c2 = 2 E B - K + 2H a^2, c0 = B^2 - a^2 K, B = a (a E - L).  For every
// r' >= r (K >= 0; r'^3 <= r'^4 / r), R(r') >= e r'^4 + c2 r'^2 + c0 with
// e = E^2 - |2H| (1 + 2 / r), and that is >= e r'^4 / 4 when
// g(u) = 3/4 e u^2 + c2 u + c0 and g'(u) are >= 0 at u = r^2 (g increases
// beyond).  R then never vanishes, so r never turns; the factor-4 margin
// dwarfs the RK4 truncation this far out.
__device__ __forceinline__ bool outbound_for_good(double r, double th, double pr, double pth, double pt,
                                                  double pphi, double a) {
    const double E = -pt, L = pphi;
    if (!(pr > 0.0) || !(E > 0.0)) return false;
    double s, c;
    sincos(safe_theta(th), &s, &c);
    const double w = L / s - a * E * s;
    const double u = r * r, a2 = a * a, cc = c * c;
    const double dlt = u - 2.0 * r + a2, sig = u + a2 * cc;
    const double P = E * (u + a2) - a * L;
    const double k0 = pth * pth + w * w;
    const double h2 = (dlt * pr * pr + k0 - P * P / dlt) / sig;  // 2H
    const double K = k0 - h2 * a2 * cc;
    const double e = E * E - fabs(h2) * (1.0 + 2.0 / r);
    if (!(K >= 0.0) || !(e > 0.0)) return false;
    const double B = a * (a * E - L);
    const double e2 = 0.75 * e, c2 = 2.0 * E * B - K + h2 * a2, c0 = B * B - a2 * K;
    return (2.0 * e2 * u + c2 >= 0.0) && ((e2 * u + c2) * u + c0 >= 0.0);
}

struct BrickTraceParams {
    const double *coeffs;        // [nr][nt][np][11]
    const double *rg, *tg, *pg;
    int nr, nt, np, max_steps, exact_step, full_trace;
    const ViewDev *view;
    double step, escape_radius, length_cm, max_tau;
    double *out;                 // [rays][4]
    double *diag;                // optional [rays][4]: optical depth, sampled segments, steps, status
};

__global__ void __launch_bounds__(128) brick_trace_kernel(const BrickTraceParams P) {
    const ViewDev &v = *P.view;
    const int64_t rays = (int64_t)v.crop_w * v.crop_h;
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ AxisHints hints;  // the brick axes' first-guess parameters (the whole block)
    load_axis_hints(hints, P.rg, P.nr, P.tg, P.nt, P.pg, P.np);
    if (r >= rays) return;
    const int px = v.x0 + (int)(r % v.crop_w), py = v.y0 + (int)(r / v.crop_w);
    double S[4] = {0.0, 0.0, 0.0, 0.0};
    double tau = 0.0;
    int steps = 0, sampled = 0, status = BHN_RAY_INVALID;
    if (v.valid) {
        const CameraRay cam = camera_ray(v, px, py);
        double y[5] = {v.r_obs, v.theta_obs, v.phi_obs, cam.pr, cam.pth};
        const double pt = cam.pt, pphi = cam.pphi, a = v.a;
        double prev_r = y[0];
        // past this radius no segment midpoint is sampled (the nonperiodic r range)
        const double r_edge = P.full_trace ? INFINITY : fmax(P.rg[0], P.rg[P.nr - 1]);
        bool stop_transfer = false;  // the optical-depth cutoff ends the integration, not the trace
        status = BHN_RAY_MAX_STEPS;
        for (int i = 1; i <= P.max_steps; ++i) {
            double yn[5];
            rk4_state(y, P.step, a, pt, pphi, yn);
            steps = i;
            if (!(isfinite(yn[0]) && isfinite(yn[1]) && isfinite(yn[2]) && isfinite(yn[3]) && isfinite(yn[4]))) {
                status = BHN_RAY_INVALID;  // kerr.py:364-366: the state is not stored
                break;
            }
            if (!stop_transfer) {
                double c[11];
                if (sample_one_hinted(P.coeffs, P.rg, P.nr, P.tg, P.nt, P.pg, P.np, hints, 0.5 * (y[0] + yn[0]),
                                      0.5 * (y[1] + yn[1]), 0.5 * (y[2] + yn[2]), c)) {
                    const double dr = yn[0] - y[0], dth = yn[1] - y[1], dph = yn[2] - y[2];
                    const double dl = sqrt((dr * dr + dth * dth) + dph * dph);
                    const double ds = fmax(P.length_cm * fmax(dl, 1.0e-14), 0.0);
                    if (P.exact_step)
                        stokes_step_exact(S, c, ds);
                    else
                        stokes_step_rk2_exact(S, c, ds);
                    tau += fmax(c[4], 0.0) * ds;
                    ++sampled;
                    if (tau >= P.max_tau) stop_transfer = true;
                }
            }
            for (int k = 0; k < 5; ++k) y[k] = yn[k];
            // kerr.py:370-378
            if (y[0] <= v.r_capture) {
                status = BHN_RAY_CAPTURED;
                break;
            }
            if (y[0] > P.escape_radius && y[0] > prev_r) {
                status = BHN_RAY_ESCAPED;
                break;
            }
            prev_r = y[0];
            if (stop_transfer) break;  // nothing after the cutoff can change the image
            // nor anything after the ray has left the brick for good: every later midpoint lies
            // beyond r_edge (r only grows from here), where the sampler returns nothing
            if (y[0] > r_edge && outbound_for_good(y[0], y[1], y[3], y[4], pt, pphi, a)) {
                status = BHN_RAY_OUTBOUND;
                break;
            }
        }
        if (stop_transfer) status = BHN_RAY_OPAQUE;
    }
    const int64_t o = v.out_offset + r;
    for (int k = 0; k < 4; ++k) P.out[4 * o + k] = isfinite(S[k]) ? S[k] : 0.0;  // nan_to_num(0, 0, 0)
    if (P.diag) {
        P.diag[4 * o + 0] = tau;
        P.diag[4 * o + 1] = sampled;
        P.diag[4 * o + 2] = steps;
        P.diag[4 * o + 3] = status;
    }
}

}  // namespace bhn

extern "C" int bhn_brick_trace_render(const double *coeffs, const double *r_grid, int32_t nr, const double *theta_grid,
                                      int32_t nt, const double *phi_grid, int32_t np, const bhn_view *view,
                                      const bhn_brick_trace_config *cfg, void *scratch, int64_t scratch_bytes,
                                      double *out, double *diag, void *stream) {
    using namespace bhn;
    if (!coeffs || !r_grid || !theta_grid || !phi_grid || !view || !cfg || !out || !scratch)
        return fail(BHN_ERR_VALUE, "missing brick, view, config or output buffer");
    if (nr < 2 || nt < 2 || np < 2) return fail(BHN_ERR_VALUE, "brick grids must contain at least 2 values");
    if (!(cfg->step > 0.0) || !std::isfinite(cfg->step)) return fail(BHN_ERR_VALUE, "step must be finite and positive");
    if (cfg->max_steps < 0) return fail(BHN_ERR_VALUE, "max_steps must be non-negative");
    if (!std::isfinite(cfg->length_cm)) return fail(BHN_ERR_VALUE, "affine-to-length scale must be finite");
    const int64_t rays = (int64_t)view->crop_w * view->crop_h;
    int rc = bhn_render_prepare(view, 1, scratch, scratch_bytes, stream);  // the view's FP64 camera tables
    if (rc) return rc;
    if (rays <= 0) return BHN_OK;
    BrickTraceParams P;
    P.coeffs = coeffs;
    P.rg = r_grid;
    P.tg = theta_grid;
    P.pg = phi_grid;
    P.nr = nr;
    P.nt = nt;
    P.np = np;
    P.max_steps = cfg->max_steps;
    P.exact_step = cfg->exact_step != 0;
    P.full_trace = cfg->full_trace != 0;
    P.view = reinterpret_cast<const ViewDev *>(static_cast<unsigned char *>(scratch) + scratch_layout(1).views);
    P.step = cfg->step;
    P.escape_radius = cfg->escape_radius;
    P.length_cm = cfg->length_cm;
    P.max_tau = cfg->max_optical_depth;
    P.out = out;
    P.diag = diag;
    brick_trace_kernel<<<(unsigned)((rays + 127) / 128), 128, 0, as_stream(stream)>>>(P);
    BHN_LAUNCH_CHECK("brick_trace_kernel");
    return BHN_OK;
}
