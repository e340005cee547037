// bhn_grrt.cuh -- the physical polarized GRRT ray loop through a GRMHD
// snapshot (FP64).  Included at the end of bhn_render.cu (camera, metric RHS).
//
// The reference renders it per pixel in Python (python/blackhole_sim/
// polarized_renderer.py:31-70): kerr.camera_ray_initial_state, then
// trace_kerr_null_geodesic (kerr.py:337-384: fixed-step RK4, every state
// stored), then integrate_polarized_kerr_grrt (polarized_transfer.py:83-145)
// over consecutive states: the snapshot sampled trilinearly at the segment
// midpoint (grmhd.py:106-121), the invariant redshift g = 1/(-p.u), the
// plasma frame with the pitch of b to the photon (synchrotron.py:104-117), the
// Hybrid coefficients at nu / g scaled by g^2 (emission) and 1/g (absorption,
// rotation), ds = L (-p.u) |d(r, theta, phi)|, and one exact or RK2 Stokes
// step, until tau reaches the cutoff.
//
// Wavefront form.  The geodesic is a long chain of dependent FP64 steps per
// ray and the coefficients are ~10^4 independent exp() evaluations per
// emitting segment, so they run as separate kernels, in rounds:
//   trace_kernel     one thread per ray: continues its RK4 geodesic until it
//                    has produced `chunk` emitting segments (or the trace
//                    ends), appending each segment's plasma frame to a list;
//   coef_kernel      one warp per listed segment: the synchrotron integrals
//                    (bhn_synchrotron.cuh) at full occupancy;
//   transfer_kernel  one thread per ray: its segments' Stokes steps in order,
//                    the optical-depth cutoff, the result when the ray ends.
// A ray whose optical depth crosses the cutoff ends at that segment (its
// trace may have run up to chunk - 1 segments further; those are discarded),
// so every result equals the segment-by-segment loop's.

#include "bhn_exact.cuh"
#include "bhn_synchrotron.cuh"
#include "bhn_transfer.cuh"

namespace bhn {

struct GrrtRay {
    double y[5], pt, pphi, prev_r;     // BL r, theta, phi, p_r, p_theta; conserved p_t, p_phi; r of the last step
    double S[4], tau, fd, gmin, gmax;  // Stokes vector, optical and Faraday depth, redshift range
    int32_t steps, valid, emit;        // RK4 steps traced, valid samples, emitting segments integrated
    int32_t trace_status;              // -1 while the geodesic is traced, then its BHN_RAY_* end
    int32_t status;                    // -1 until the ray's result is written
    int32_t count;                     // emitting segments listed in this round
};

struct SegIn {    // one emitting segment's plasma frame (the coefficient kernel's input)
    double n_e, te, b, cos_los, chi, nu_emit, jf, kf;
};
struct SegSide {  // what the transfer needs besides the coefficients
    double ds, g;
    int32_t step, valid;
};

struct WaveState {
    GrrtRay *ray;               // [rays]
    SegIn *seg;                 // [rays * chunk], in append order
    SegSide *side;              // [rays][chunk]
    int32_t *slot;              // [rays][chunk]: index of the ray's k-th segment in seg / coef
    double *coef;               // [rays * chunk][12]: scaled coefficients
    unsigned long long *n_seg;  // segments listed in this round
    int64_t rays;
    int32_t chunk;
};

struct TraceParams {
    const double *fields;       // [nr][nt][np][11]: rho, Theta_e, pressure, b^mu (4), u^mu (4)
    const double *rg, *tg, *pg;
    int nr, nt, np, max_steps;
    const ViewDev *view;
    double step, escape_radius, nu, length_cm, min_redshift, flux_scale, rho_unit, b_unit, mu_e_mp;
    int full_trace;             // 0: a ray past the snapshot's outer radius, moving out for good, ends there
    WaveState W;
};
struct CoefParams {
    synch::Model M;
    WaveState W;
};
struct TransferParams {
    const ViewDev *view;
    double max_tau;
    int exact_step;
    double *out;                // [rays][4] Stokes
    double *diag;               // optional [rays][8]: tau, emit, valid, faraday depth, g min, g max, steps, status
    WaveState W;
};

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

__device__ __forceinline__ void rk4_state(const double y[5], double h, double a, double pt, double pphi, double yn[5]) {
    // kerr.py:306-313 on (r, theta, phi, p_r, p_theta)
    Deriv64 k1, k2, k3, k4;
    const double hh = 0.5 * h;
    rhs64(y[0], y[1], y[3], y[4], pt, pphi, a, k1);
    rhs64(y[0] + hh * k1.r, y[1] + hh * k1.th, y[3] + hh * k1.pr, y[4] + hh * k1.pth, pt, pphi, a, k2);
    rhs64(y[0] + hh * k2.r, y[1] + hh * k2.th, y[3] + hh * k2.pr, y[4] + hh * k2.pth, pt, pphi, a, k3);
    rhs64(y[0] + h * k3.r, y[1] + h * k3.th, y[3] + h * k3.pr, y[4] + h * k3.pth, pt, pphi, a, k4);
    const double h6 = h / 6.0;
    yn[0] = y[0] + h6 * (((k1.r + 2.0 * k2.r) + 2.0 * k3.r) + k4.r);
    yn[1] = safe_theta(y[1] + h6 * (((k1.th + 2.0 * k2.th) + 2.0 * k3.th) + k4.th));
    yn[2] = y[2] + h6 * (((k1.ph + 2.0 * k2.ph) + 2.0 * k3.ph) + k4.ph);
    yn[3] = y[3] + h6 * (((k1.pr + 2.0 * k2.pr) + 2.0 * k3.pr) + k4.pr);
    yn[4] = y[4] + h6 * (((k1.pth + 2.0 * k2.pth) + 2.0 * k3.pth) + k4.pth);
}

__device__ __forceinline__ void write_result(const ViewDev &v, int64_t ray, const GrrtRay &R, int status,
                                             double *out, double *diag) {
    const int64_t o = v.out_offset + ray;  // the crop's rays in row order
    for (int k = 0; k < 4; ++k) out[4 * o + k] = R.S[k];
    if (diag) {
        double *d = diag + 8 * o;
        d[0] = R.tau;
        d[1] = R.emit;
        d[2] = R.valid;
        d[3] = R.fd;
        d[4] = R.gmin < INFINITY ? R.gmin : 0.0;
        d[5] = R.gmax;
        d[6] = R.steps;
        d[7] = status;
    }
}

__global__ void __launch_bounds__(128) grrt_init_kernel(const TraceParams P, double *out, double *diag) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.W.rays) return;
    const ViewDev &v = *P.view;
    GrrtRay &R = P.W.ray[r];
    const int px = v.x0 + (int)(r % v.crop_w), py = v.y0 + (int)(r / v.crop_w);
    const CameraRay cam = camera_ray(v, px, py);
    R.y[0] = v.r_obs;
    R.y[1] = v.theta_obs;
    R.y[2] = v.phi_obs;
    R.y[3] = cam.pr;
    R.y[4] = cam.pth;
    R.pt = cam.pt;
    R.pphi = cam.pphi;
    R.prev_r = v.r_obs;
    for (int k = 0; k < 4; ++k) R.S[k] = 0.0;
    R.tau = R.fd = R.gmax = 0.0;
    R.gmin = INFINITY;
    R.steps = R.valid = R.emit = R.count = 0;
    R.trace_status = -1;
    R.status = -1;
    if (!v.valid) {
        R.status = BHN_RAY_INVALID;
        write_result(v, r, R, BHN_RAY_INVALID, out, diag);
    }
}

__global__ void __launch_bounds__(128) grrt_trace_kernel(const TraceParams P) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ AxisHints hints;  // the snapshot axes' first-guess parameters (the whole block)
    load_axis_hints(hints, P.rg, P.nr, P.tg, P.nt, P.pg, P.np);
    if (r >= P.W.rays) return;
    GrrtRay &R = P.W.ray[r];
    R.count = 0;
    if (R.status >= 0 || R.trace_status >= 0) return;
    const ViewDev &v = *P.view;
    const double a = v.a, pt = R.pt, pphi = R.pphi;
    const double r_edge = P.full_trace ? INFINITY : fmax(hints.g0[0], hints.gn[0]);
    double y[5] = {R.y[0], R.y[1], R.y[2], R.y[3], R.y[4]};
    double prev_r = R.prev_r;
    int steps = R.steps, valid = R.valid, count = 0, ts = -1;
    SegSide *side = P.W.side + r * P.W.chunk;
    int32_t *slot = P.W.slot + r * P.W.chunk;
    for (;;) {
        if (steps >= P.max_steps) {
            ts = BHN_RAY_MAX_STEPS;
            break;
        }
        double yn[5];
        rk4_state(y, P.step, a, pt, pphi, yn);
        ++steps;
        if (!(isfinite(yn[0]) && isfinite(yn[1]) && isfinite(yn[2]) && isfinite(yn[3]) && isfinite(yn[4]))) {
            ts = BHN_RAY_INVALID;  // kerr.py:364-366: not stored, no segment
            break;
        }
        // segment (y, yn): polarized_transfer.py:103-143
        const double mr = 0.5 * (y[0] + yn[0]), mth = 0.5 * (y[1] + yn[1]), mph = 0.5 * (y[2] + yn[2]);
        const double mpr = 0.5 * (y[3] + yn[3]), mpth = 0.5 * (y[4] + yn[4]);
        double f[11];
        const bool inside = isfinite(mr) && isfinite(mth) && isfinite(mph) &&
                            sample_one_hinted(P.fields, P.rg, P.nr, P.tg, P.nt, P.pg, P.np, hints, mr, mth, mph, f);
        // grmhd.py:119-120: rho > 0, Theta_e > 0, finite u
        if (inside && f[0] > 0.0 && f[1] > 0.0 && isfinite(f[7]) && isfinite(f[8]) && isfinite(f[9]) &&
            isfinite(f[10])) {
            ++valid;
            // radiative_transfer.py:91-99
            const double e_emit = -(((pt * f[7] + mpr * f[8]) + mpth * f[9]) + pphi * f[10]);
            const double g = (e_emit > 0.0 && isfinite(e_emit)) ? 1.0 / e_emit : 0.0;
            if (g >= P.min_redshift) {
                // synchrotron.py:104-117 with calibration.py:113-119
                const double b1 = f[4], b2 = f[5], b3 = f[6];
                const double b_code = sqrt((b1 * b1 + b2 * b2) + b3 * b3);
                SegIn s;
                s.n_e = f[0] * P.rho_unit / P.mu_e_mp;
                s.cos_los = 0.0;
                if (b_code > 0.0) {
                    const double nk = sqrt((mpr * mpr + mpth * mpth) + pphi * pphi);
                    if (nk > 0.0)
                        s.cos_los = fmin(fmax(((b1 * mpr + b2 * mpth) + b3 * pphi) / (b_code * nk), -1.0), 1.0);
                }
                s.chi = b_code > 0.0 ? atan2(b3, b2) : 0.0;
                s.te = fmax(f[1], 1.0e-8);
                s.b = fmax(b_code * P.b_unit, 0.0);
                s.nu_emit = P.nu / g;
                s.jf = g * g * P.flux_scale;
                s.kf = 1.0 / fmax(g, 1.0e-300);
                const double dr = yn[0] - y[0], dth = yn[1] - y[1], dph = yn[2] - y[2];
                const double dl = sqrt((dr * dr + dth * dth) + dph * dph);
                SegSide sd;
                sd.ds = P.length_cm * fmax(e_emit, 0.0) * fmax(dl, 1.0e-14);
                sd.g = g;
                sd.step = steps;
                sd.valid = valid;
                const unsigned long long idx = atomicAdd(P.W.n_seg, 1ull);
                P.W.seg[idx] = s;
                side[count] = sd;
                slot[count] = (int32_t)idx;
                ++count;
            }
        }
        for (int k = 0; k < 5; ++k) y[k] = yn[k];
        // kerr.py:370-378
        if (y[0] <= v.r_capture) {
            ts = BHN_RAY_CAPTURED;
            break;
        }
        if (y[0] > P.escape_radius && y[0] > prev_r) {
            ts = BHN_RAY_ESCAPED;
            break;
        }
        prev_r = y[0];
        // past the snapshot's outer radius for good: every later midpoint lies outside it (no segment)
        if (y[0] > r_edge && outbound_for_good(y[0], y[1], y[3], y[4], pt, pphi, a)) {
            ts = BHN_RAY_OUTBOUND;
            break;
        }
        if (count == P.W.chunk) break;  // this round's list is full: continue in the next round
    }
    for (int k = 0; k < 5; ++k) R.y[k] = y[k];
    R.prev_r = prev_r;
    R.steps = steps;
    R.valid = valid;
    R.count = count;
    R.trace_status = ts;
}

// One warp per listed segment (a persistent grid over this round's list).
__global__ void __launch_bounds__(128, 6) grrt_coef_kernel(const __grid_constant__ CoefParams P) {
    __shared__ synch::TableSmem T;
    synch::load_table(T, P.M);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const unsigned long long n = *P.W.n_seg;
    const unsigned long long warps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long i = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const SegIn s = P.W.seg[i];
        double c[11];
        synch::coefficients(T, P.M, s.n_e, s.te, s.b, s.cos_los, s.chi, s.nu_emit, c);
        double *o = P.W.coef + 12 * i;
#pragma unroll
        for (int k = 0; k < 11; ++k)
            if (lane == k) o[k] = c[k] * (k < 4 ? s.jf : s.kf);
    }
}

__global__ void __launch_bounds__(128) grrt_transfer_kernel(const TransferParams P) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *P.W.n_seg = 0;  // the coefficient kernel has read it
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.W.rays) return;
    GrrtRay &R = P.W.ray[r];
    if (R.status >= 0) return;
    const SegSide *side = P.W.side + r * P.W.chunk;
    const int32_t *slot = P.W.slot + r * P.W.chunk;
    double S[4] = {R.S[0], R.S[1], R.S[2], R.S[3]};
    double tau = R.tau, fd = R.fd, gmin = R.gmin, gmax = R.gmax;
    int emit = R.emit, status = -1;
    for (int k = 0; k < R.count; ++k) {
        const SegSide sd = side[k];
        const double *cp = P.W.coef + 12 * (int64_t)slot[k];
        double c[11];
        for (int q = 0; q < 11; ++q) c[q] = cp[q];
        if (P.exact_step)
            stokes_step_exact(S, c, sd.ds);
        else
            stokes_step_rk2_exact(S, c, sd.ds);
        tau = tau + fmax(c[4], 0.0) * sd.ds;
        fd = fd + (fabs(c[8]) + fabs(c[9]) + fabs(c[10])) * sd.ds;
        ++emit;
        gmin = fmin(gmin, sd.g);
        gmax = fmax(gmax, sd.g);
        if (tau >= P.max_tau) {  // polarized_transfer.py:141-142: the ray ends at this segment
            status = BHN_RAY_OPAQUE;
            R.steps = sd.step;
            R.valid = sd.valid;
            break;
        }
    }
    for (int q = 0; q < 4; ++q) R.S[q] = S[q];
    R.tau = tau;
    R.fd = fd;
    R.gmin = gmin;
    R.gmax = gmax;
    R.emit = emit;
    if (status < 0) status = R.trace_status;
    if (status >= 0) {
        R.status = status;
        write_result(*P.view, r, R, status, P.out, P.diag);
    }
}

struct GrrtLayout {
    int64_t views, n_seg, ray, seg, side, slot, coef, total;
};
inline GrrtLayout grrt_layout(int64_t rays, int64_t chunk) {
    auto up = [](int64_t x) { return (x + 255) & ~(int64_t)255; };
    GrrtLayout L;
    L.views = 0;
    L.n_seg = up(scratch_layout(1).total);
    L.ray = L.n_seg + 256;
    L.seg = up(L.ray + rays * (int64_t)sizeof(GrrtRay));
    L.side = up(L.seg + rays * chunk * (int64_t)sizeof(SegIn));
    L.slot = up(L.side + rays * chunk * (int64_t)sizeof(SegSide));
    L.coef = up(L.slot + rays * chunk * 4);
    L.total = up(L.coef + rays * chunk * 12 * 8);
    return L;
}
constexpr int64_t kGrrtMaxChunk = 4096;

}  // namespace bhn

extern "C" int64_t bhn_grrt_scratch_bytes(int64_t rays, int32_t chunk) {
    if (rays < 0 || chunk < 1) return -1;
    return bhn::grrt_layout(rays, chunk).total;
}

extern "C" int bhn_grrt_render(const double *fields, const double *r_grid, int32_t nr, const double *theta_grid,
                               int32_t nt, const double *phi_grid, int32_t np, const bhn_view *view,
                               const bhn_synchrotron_model *model, const bhn_grrt_config *cfg, void *scratch,
                               int64_t scratch_bytes, double *out, double *diag, void *stream) {
    using namespace bhn;
    if (!fields || !r_grid || !theta_grid || !phi_grid || !view || !cfg || !out || !scratch)
        return fail(BHN_ERR_VALUE, "missing snapshot, view, config or output buffer");
    if (nr < 2 || nt < 2 || np < 2) return fail(BHN_ERR_VALUE, "snapshot grids must contain at least 2 values");
    if (!(cfg->step > 0.0) || !std::isfinite(cfg->step)) return fail(BHN_ERR_VALUE, "step must be finite and positive");
    if (cfg->max_steps < 0) return fail(BHN_ERR_VALUE, "max_steps must be non-negative");
    if (!(cfg->nu_hz > 0.0) || !std::isfinite(cfg->nu_hz)) return fail(BHN_ERR_VALUE, "observing frequency must be positive");
    if (!(cfg->length_cm > 0.0) || !std::isfinite(cfg->length_cm))
        return fail(BHN_ERR_VALUE, "affine-to-length scale must be finite and positive");
    const int64_t rays = (int64_t)view->crop_w * view->crop_h;
    if (rays <= 0) return BHN_OK;
    // the largest chunk the scratch holds
    int64_t chunk = 0;
    for (int64_t lo = 1, hi = kGrrtMaxChunk; lo <= hi;) {
        const int64_t mid = (lo + hi) / 2;
        if (grrt_layout(rays, mid).total <= scratch_bytes) {
            chunk = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (chunk < 1)
        return fail(BHN_ERR_VALUE, "scratch too small: bhn_grrt_scratch_bytes(rays, 1) = " +
                                       std::to_string(grrt_layout(rays, 1).total) + " bytes");
    static CoefParams C;  // ~10 KB (the model's tables): kept off the host stack; filled under the lock
    static std::mutex lock;
    std::lock_guard<std::mutex> g(lock);
    int rc = synch::fill_model(model, C.M);
    if (rc) return rc;
    rc = bhn_render_prepare(view, 1, scratch, scratch_layout(1).total, stream);  // FP64 camera tables of the view
    if (rc) return rc;
    const GrrtLayout GL = grrt_layout(rays, chunk);
    unsigned char *sc = reinterpret_cast<unsigned char *>(scratch);
    WaveState W;
    W.ray = reinterpret_cast<GrrtRay *>(sc + GL.ray);
    W.seg = reinterpret_cast<SegIn *>(sc + GL.seg);
    W.side = reinterpret_cast<SegSide *>(sc + GL.side);
    W.slot = reinterpret_cast<int32_t *>(sc + GL.slot);
    W.coef = reinterpret_cast<double *>(sc + GL.coef);
    W.n_seg = reinterpret_cast<unsigned long long *>(sc + GL.n_seg);
    W.rays = rays;
    W.chunk = (int32_t)chunk;
    C.W = W;
    const ViewDev *vd = reinterpret_cast<const ViewDev *>(sc + scratch_layout(1).views);
    TraceParams T;
    T.fields = fields;
    T.rg = r_grid;
    T.tg = theta_grid;
    T.pg = phi_grid;
    T.nr = nr;
    T.nt = nt;
    T.np = np;
    T.max_steps = cfg->max_steps;
    T.full_trace = cfg->full_trace != 0;
    T.view = vd;
    T.step = cfg->step;
    T.escape_radius = cfg->escape_radius;
    T.nu = cfg->nu_hz;
    T.length_cm = cfg->length_cm;
    T.min_redshift = cfg->min_redshift;
    T.flux_scale = cfg->flux_scale;
    T.rho_unit = C.M.rho_unit;
    T.b_unit = C.M.b_unit;
    T.mu_e_mp = C.M.mu_e_mp;
    T.W = W;
    TransferParams X;
    X.view = vd;
    X.max_tau = cfg->max_optical_depth;
    X.exact_step = cfg->exact_step != 0;
    X.out = out;
    X.diag = diag;
    X.W = W;
    int dev = 0, sms = 148, per_sm = 0;
    BHN_CUDA_TRY(cudaGetDevice(&dev));
    BHN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BHN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grrt_coef_kernel, 128, 0));
    cudaStream_t s = as_stream(stream);
    const unsigned ray_blocks = (unsigned)((rays + 127) / 128);
    const unsigned coef_blocks = (unsigned)std::min<int64_t>((rays * chunk + 3) / 4, (int64_t)sms * std::max(per_sm, 1));
    BHN_CUDA_TRY(cudaMemsetAsync(W.n_seg, 0, sizeof(unsigned long long), s));
    grrt_init_kernel<<<ray_blocks, 128, 0, s>>>(T, out, diag);
    BHN_LAUNCH_CHECK("grrt_init_kernel");
    // every round either ends a ray's trace or lists chunk segments of it, one step each at least
    const int64_t rounds = (int64_t)cfg->max_steps / chunk + 2;
    for (int64_t k = 0; k < rounds; ++k) {
        grrt_trace_kernel<<<ray_blocks, 128, 0, s>>>(T);
        BHN_LAUNCH_CHECK("grrt_trace_kernel");
        grrt_coef_kernel<<<coef_blocks, 128, 0, s>>>(C);
        BHN_LAUNCH_CHECK("grrt_coef_kernel");
        grrt_transfer_kernel<<<ray_blocks, 128, 0, s>>>(X);
        BHN_LAUNCH_CHECK("grrt_transfer_kernel");
    }
    return BHN_OK;
}
