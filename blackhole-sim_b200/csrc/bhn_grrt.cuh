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
// One warp owns a ray: all 32 lanes step the geodesic identically (it is cheap
// next to the coefficients), and the warp evaluates each segment's
// synchrotron integrals together (bhn_synchrotron.cuh).  Segments are
// integrated as the ray is traced; the trace's own stopping rules end it.

#include "bhn_exact.cuh"
#include "bhn_synchrotron.cuh"
#include "bhn_transfer.cuh"

namespace bhn {

struct GrrtParams {
    synch::Model M;
    const double *fields;       // [nr][nt][np][11]: rho, Theta_e, pressure, b^mu (4), u^mu (4)
    const double *rg, *tg, *pg;
    int nr, nt, np;
    const ViewDev *view;
    double step, escape_radius, nu, length_cm, max_tau, min_redshift, flux_scale;
    int max_steps, exact_step;
    double *out;                // [rays][4] Stokes
    double *diag;               // optional [rays][8]: tau, emit, valid, faraday depth, g min, g max, steps, status
    unsigned long long *queue;  // next ray to hand out (zeroed before the launch)
};

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

// The state a ray carries across its segments, one copy per warp in shared
// memory: the lanes hold identical values (they run the same arithmetic, and
// the butterfly sums of the coefficient integrals give every lane the same
// bits), so every lane stores and reloads the same numbers.  Keeping it out of
// registers while the warp evaluates a segment's synchrotron integrals leaves
// those registers to the integrals.
struct RayState {
    double y[5], S[4], tau, fd, gmin, gmax, prev_r, pt, pphi;
};

__global__ void __launch_bounds__(128, 4) grrt_kernel(const __grid_constant__ GrrtParams P) {
    __shared__ synch::TableSmem T;
    __shared__ RayState ray_state[4];
    synch::load_table(T, P.M);
    __syncthreads();
    const ViewDev &v = *P.view;
    const int lane = threadIdx.x & 31;
    volatile RayState &st = ray_state[threadIdx.x >> 5];
    const int64_t rays = (int64_t)v.crop_w * v.crop_h;
    // Rays differ by orders of magnitude in emitting segments: a persistent
    // grid whose warps take the next ray from one counter keeps every warp busy
    // until the last rays.
    for (;;) {
        unsigned long long next = 0;
        if (lane == 0) next = atomicAdd(P.queue, 1ull);
        const int64_t ray = (int64_t)__shfl_sync(0xffffffffu, next, 0);
        if (ray >= rays) break;
        const int px = v.x0 + (int)(ray % v.crop_w), py = v.y0 + (int)(ray / v.crop_w);
        {
            const CameraRay cam = camera_ray(v, px, py);
            st.y[0] = v.r_obs;
            st.y[1] = v.theta_obs;
            st.y[2] = v.phi_obs;
            st.y[3] = cam.pr;
            st.y[4] = cam.pth;
            st.pt = cam.pt;
            st.pphi = cam.pphi;
            for (int k = 0; k < 4; ++k) st.S[k] = 0.0;
            st.tau = 0.0;
            st.fd = 0.0;
            st.gmin = INFINITY;
            st.gmax = 0.0;
            st.prev_r = v.r_obs;
        }
        int emit = 0, valid = 0, steps = 0, status = v.valid ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID;
        for (int i = 1; i <= P.max_steps && v.valid; ++i) {
            const double a = v.a, pt = st.pt, pphi = st.pphi;
            double y[5], yn[5];
            for (int k = 0; k < 5; ++k) y[k] = st.y[k];
            rk4_state(y, P.step, a, pt, pphi, yn);
            steps = i;
            if (!(isfinite(yn[0]) && isfinite(yn[1]) && isfinite(yn[2]) && isfinite(yn[3]) && isfinite(yn[4]))) {
                status = BHN_RAY_INVALID;  // kerr.py:364-366: not stored, no segment
                break;
            }
            for (int k = 0; k < 5; ++k) st.y[k] = yn[k];
            // segment (y, yn): polarized_transfer.py:103-143
            const double mr = 0.5 * (y[0] + yn[0]), mth = 0.5 * (y[1] + yn[1]), mph = 0.5 * (y[2] + yn[2]);
            const double mpr = 0.5 * (y[3] + yn[3]), mpth = 0.5 * (y[4] + yn[4]);
            double f[11];
            const bool inside = isfinite(mr) && isfinite(mth) && isfinite(mph) &&
                                sample_one_exact(P.fields, P.rg, P.nr, P.tg, P.nt, P.pg, P.np, mr, mth, mph, f);
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
                    const double n_e = f[0] * P.M.rho_unit / P.M.mu_e_mp;
                    double cos_los = 0.0;
                    if (b_code > 0.0) {
                        const double nk = sqrt((mpr * mpr + mpth * mpth) + pphi * pphi);
                        if (nk > 0.0)
                            cos_los = fmin(fmax(((b1 * mpr + b2 * mpth) + b3 * pphi) / (b_code * nk), -1.0), 1.0);
                    }
                    const double chi = b_code > 0.0 ? atan2(b3, b2) : 0.0;
                    const double te = fmax(f[1], 1.0e-8), b = fmax(b_code * P.M.b_unit, 0.0);
                    const double jf = g * g * P.flux_scale, kf = 1.0 / fmax(g, 1.0e-300);
                    const double dr = yn[0] - y[0], dth = yn[1] - y[1], dph = yn[2] - y[2];
                    const double dl = sqrt((dr * dr + dth * dth) + dph * dph);
                    const double ds = P.length_cm * fmax(e_emit, 0.0) * fmax(dl, 1.0e-14);
                    st.gmin = fmin(st.gmin, g);
                    st.gmax = fmax(st.gmax, g);
                    double c[11];
                    synch::coefficients(T, P.M, n_e, te, b, cos_los, chi, P.nu / g, c);
#pragma unroll
                    for (int k = 0; k < 4; ++k) c[k] *= jf;
#pragma unroll
                    for (int k = 4; k < 11; ++k) c[k] *= kf;
                    double S[4];
                    for (int k = 0; k < 4; ++k) S[k] = st.S[k];
                    if (P.exact_step)
                        stokes_step_exact(S, c, ds);
                    else
                        stokes_step_rk2_exact(S, c, ds);
                    for (int k = 0; k < 4; ++k) st.S[k] = S[k];
                    const double tau = st.tau + fmax(c[4], 0.0) * ds;
                    st.tau = tau;
                    st.fd = st.fd + (fabs(c[8]) + fabs(c[9]) + fabs(c[10])) * ds;
                    ++emit;
                    if (tau >= P.max_tau) {
                        status = BHN_RAY_OPAQUE;
                        break;
                    }
                }
            }
            // kerr.py:370-378
            const double r = st.y[0];
            if (r <= v.r_capture) {
                status = BHN_RAY_CAPTURED;
                break;
            }
            if (r > P.escape_radius && r > st.prev_r) {
                status = BHN_RAY_ESCAPED;
                break;
            }
            st.prev_r = r;
        }
        if (lane == 0) {
            const int64_t o = v.out_offset + (int64_t)(py - v.y0) * v.crop_w + (px - v.x0);
            for (int k = 0; k < 4; ++k) P.out[4 * o + k] = st.S[k];
            if (P.diag) {
                double *d = P.diag + 8 * o;
                d[0] = st.tau;
                d[1] = emit;
                d[2] = valid;
                d[3] = st.fd;
                d[4] = st.gmin < INFINITY ? st.gmin : 0.0;
                d[5] = st.gmax;
                d[6] = steps;
                d[7] = status;
            }
        }
        __syncwarp();  // every lane is done with this ray's state before the next ray overwrites it
    }
}

}  // namespace bhn

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
    static GrrtParams P;  // ~10 KB: kept off the host stack; filled under the lock
    static std::mutex lock;
    std::lock_guard<std::mutex> g(lock);
    int rc = synch::fill_model(model, P.M);
    if (rc) return rc;
    rc = bhn_render_prepare(view, 1, scratch, scratch_bytes, stream);  // FP64 camera tables of the view
    if (rc) return rc;
    const ScratchLayout L = scratch_layout(1);
    unsigned char *sc = reinterpret_cast<unsigned char *>(scratch);
    P.fields = fields;
    P.rg = r_grid;
    P.tg = theta_grid;
    P.pg = phi_grid;
    P.nr = nr;
    P.nt = nt;
    P.np = np;
    P.view = reinterpret_cast<const ViewDev *>(sc + L.views);
    P.step = cfg->step;
    P.escape_radius = cfg->escape_radius;
    P.nu = cfg->nu_hz;
    P.length_cm = cfg->length_cm;
    P.max_tau = cfg->max_optical_depth;
    P.min_redshift = cfg->min_redshift;
    P.flux_scale = cfg->flux_scale;
    P.max_steps = cfg->max_steps;
    P.exact_step = cfg->exact_step != 0;
    P.out = out;
    P.diag = diag;
    const int64_t rays = (int64_t)view->crop_w * view->crop_h;
    if (rays <= 0) return BHN_OK;
    int dev = 0, sms = 148, per_sm = 0;
    BHN_CUDA_TRY(cudaGetDevice(&dev));
    BHN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BHN_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grrt_kernel, 128, 0));
    const int64_t blocks = std::min<int64_t>((rays + 3) / 4, (int64_t)sms * std::max(per_sm, 1));
    P.queue = reinterpret_cast<unsigned long long *>(sc + L.queue);
    BHN_CUDA_TRY(cudaMemsetAsync(P.queue, 0, sizeof(unsigned long long), as_stream(stream)));
    grrt_kernel<<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(P);
    BHN_LAUNCH_CHECK("grrt_kernel");
    return BHN_OK;
}
