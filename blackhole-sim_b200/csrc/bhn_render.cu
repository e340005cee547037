// bhn_render.cu -- the fused persistent GRRT ray kernel.
//
// One kernel does, per ray (accelerated_renderer.py:129-150):
//   camera ray (kerr.py:188-233, FP64)
//   -> RK2 midpoint steps of the Kerr null geodesic (kerr.py:285-303 right-hand
//      side, native/cuda/kerr_stokes_kernel.cu:13 step form, h = clamp(h_scale r))
//   -> termination tests of kerr.py:371-377 (FP64)
//   -> per-segment midpoint brick gather with the nonperiodic valid mask
//      (accelerated_renderer.py:113-118, native_kernels.py:137-186)
//   -> Stokes RK2 step, optical depth, cutoff (accelerated_renderer.py:119-126)
// with all ray state in registers.  Work distribution: a persistent grid pulls
// ray slots from one global queue head; each warp refills its finished lanes
// with a single atomicAdd (ballot + popc ray compaction, the persistent-thread
// scheme of Aila & Laine, "Understanding the efficiency of ray traversal on
// GPUs", HPG 2009), so uneven ray lengths do not idle whole warps.
//
// Two tracers share that loop:
//   Tracer32 -- the product kernel: geodesic and transfer in FP32; positions
//               (r, theta, phi) accumulate in FP64, which keeps the horizon and
//               turning-point tests and the pole distance of the metric inverse
//               in FP64; camera momenta are normalised in FP64.
//   Tracer64 -- FP64 throughout with the reference's own formulation of the
//               right-hand side; the GPU form of the CPU oracle, used for the
//               fine-step precision study on images too large for the CPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "bhn_internal.cuh"

namespace bhn {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------ view set-up
__device__ __forceinline__ double safe_theta(double th) {  // kerr.py:35-36
    return fmin(fmax(th, kEpsTheta), kPi - kEpsTheta);
}

__global__ void setup_views_kernel(const bhn_view *__restrict__ raw, int n, ViewDev *__restrict__ views,
                                   int64_t *__restrict__ ray_begin, QueueState *q) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        bhn_view v = raw[i];
        ViewDev d;
        memset(&d, 0, sizeof d);
        const double a = v.spin_a, r = v.r_obs, th = safe_theta(v.theta_obs);
        const double deg = kPi / 180.0;
        const double ct = cos(th), st = sin(th);
        // kerr.py:52-64
        const double sig = r * r + a * a * (ct * ct);
        const double dlt = r * r - 2.0 * r + a * a;
        const double s2 = st * st;
        const double A = (r * r + a * a) * (r * r + a * a) - a * a * dlt * s2;
        d.valid = (dlt > 0.0) && (fabs(st) >= kEpsTheta) && (fabs(a) < 1.0) && (v.width > 0) && (v.height > 0);
        d.a = a;
        d.r_obs = r;
        d.theta_obs = th;
        d.phi_obs = v.phi_obs;
        // kerr.py:67-83 (covariant) and :86-102 (contravariant)
        d.gcov00 = -(1.0 - 2.0 * r / sig);
        d.gcov03 = -2.0 * a * r * s2 / sig;
        d.gcov11 = sig / dlt;
        d.gcov22 = sig;
        d.gcov33 = A * s2 / sig;
        const double s2c = fmax(s2, kEpsTheta * kEpsTheta);
        d.gcon00 = -A / (sig * dlt);
        d.gcon03 = -2.0 * a * r / (sig * dlt);
        d.gcon11 = dlt / sig;
        d.gcon22 = 1.0 / sig;
        d.gcon33 = (dlt - a * a * s2c) / (sig * dlt * s2c);
        // kerr.py:141-148 ZAMO tetrad
        const double lapse = sqrt(sig * dlt / A);
        const double omega = 2.0 * a * r / A;
        d.pt_con = 1.0 / lapse;
        d.pphi_con0 = omega / lapse;
        d.e_r = sqrt(dlt / sig);
        d.e_th = 1.0 / sqrt(sig);
        d.e_ph = 1.0 / sqrt(d.gcov33);
        // kerr.py:208-223 image plane
        const double aspect = (double)v.width / (double)v.height;
        d.tan_y = tan(0.5 * (v.fov_y_deg * deg));
        d.tan_x = aspect * d.tan_y;
        d.has_roll = v.roll_deg != 0.0;
        d.cos_roll = cos(v.roll_deg * deg);
        d.sin_roll = sin(v.roll_deg * deg);
        d.width_d = (double)v.width;
        d.height_d = (double)v.height;
        d.r_plus = 1.0 + sqrt(1.0 - a * a);   // kerr.py:39-42
        d.r_minus = 1.0 - sqrt(1.0 - a * a);
        d.r_capture = d.r_plus * (1.0 + 2.0e-4);  // kerr.py:371
        d.escape_radius = v.escape_radius;
        d.h_scale = v.h_scale;
        d.h_min = v.h_min;
        d.h_max = v.h_max;
        d.L = v.affine_to_length_cm;
        d.max_tau = v.max_optical_depth;
        d.width = v.width;
        d.height = v.height;
        d.x0 = v.x0;
        d.y0 = v.y0;
        d.crop_w = v.crop_w;
        d.crop_h = v.crop_h;
        d.max_steps = v.max_steps;
        d.out_offset = v.out_offset;
        d.ray_count = (int64_t)v.crop_w * v.crop_h;
        views[i] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t acc = 0;
        for (int i = 0; i < n; ++i) {
            views[i].ray_begin = acc;
            ray_begin[i] = acc;
            acc += views[i].ray_count;
        }
        ray_begin[n] = acc;
        q->total = (unsigned long long)acc;
        q->n_views = (uint32_t)n;
    }
}

// ------------------------------------------------------------ shared pieces
struct PixelRef {
    int32_t px, py;      // absolute pixel
    int64_t out_idx;     // index into the output image buffer
};

// Ray k of a view's crop in tile order: bands of tile_h rows, tiles of tile_w
// columns inside a band (the last band / tile of a band may be narrower).
__device__ __forceinline__ PixelRef pixel_of(const ViewDev &v, int64_t k, int tw, int th) {
    const int cw = v.crop_w, ch = v.crop_h;
    const int kk = (int)k;
    const int band_rays = th * cw;
    const int band = kk / band_rays;
    const int kb = kk - band * band_rays;
    const int bh = min(th, ch - band * th);
    const int tile = kb / (tw * bh);
    const int kt = kb - tile * tw * bh;
    const int tw_eff = min(tw, cw - tile * tw);
    const int lx = tile * tw + kt % tw_eff;
    const int ly = band * th + kt / tw_eff;
    PixelRef p;
    p.px = v.x0 + lx;
    p.py = v.y0 + ly;
    p.out_idx = v.out_offset + (int64_t)ly * cw + lx;
    return p;
}

// kerr.py:188-233 for pixel (px, py) of a view: returns covariant momenta and
// |H0| (kerr.py:352), all in FP64.
struct CameraRay {
    double pt, pr, pth, pphi, H0;
};
__device__ __forceinline__ CameraRay camera_ray(const ViewDev &v, int px, int py) {
    // accelerated_renderer.py:136-140
    const double ndc_y = 1.0 - 2.0 * ((double)py + 0.5) / v.height_d;
    const double ndc_x = 2.0 * ((double)px + 0.5) / v.width_d - 1.0;
    double n0 = -1.0, n1 = -ndc_y * v.tan_y, n2 = ndc_x * v.tan_x;
    if (v.has_roll) {
        const double t1 = v.cos_roll * n1 - v.sin_roll * n2;
        const double t2 = v.sin_roll * n1 + v.cos_roll * n2;
        n1 = t1;
        n2 = t2;
    }
    const double nn = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    n0 /= nn;
    n1 /= nn;
    n2 /= nn;
    const double pct = v.pt_con, pcr = n0 * v.e_r, pcth = n1 * v.e_th, pcph = v.pphi_con0 + n2 * v.e_ph;
    CameraRay c;
    c.pt = v.gcov00 * pct + v.gcov03 * pcph;
    c.pr = v.gcov11 * pcr;
    c.pth = v.gcov22 * pcth;
    c.pphi = v.gcov03 * pct + v.gcov33 * pcph;
    const double H = 0.5 * (v.gcon00 * c.pt * c.pt + 2.0 * v.gcon03 * c.pt * c.pphi + v.gcon11 * c.pr * c.pr +
                            v.gcon22 * c.pth * c.pth + v.gcon33 * c.pphi * c.pphi);
    c.H0 = fabs(H);
    return c;
}

struct LaneCounters {
    unsigned long long steps, brick;
    uint32_t rays, status[5];
    float max_drift, max_drift_escaped;
};

struct RenderParams {
    const void *records;
    const void *tables;
    int nr, nt, np, n_views;
    const ViewDev *views;
    const int64_t *ray_begin;
    QueueState *q;
    bhn_render_stats *stats;
    void *out;
    int32_t *ray_steps;
    uint8_t *ray_status;
    float *ray_drift;
    int tile_w, tile_h, refill_min;
    int tables_bytes;
};

__device__ __forceinline__ int find_view(const int64_t *begin, int n, int64_t slot) {
    int lo = 0, hi = n;  // largest i with begin[i] <= slot
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (begin[mid] <= slot) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------ FP32 tracer
// sin and cos on [0, pi/2] by their Taylor series (through x^11 and x^12; the
// truncation error is below 6e-8 at pi/2), evaluated by Horner in x^2.
__device__ __forceinline__ void sincos_quadrant(float x, float &s, float &c) {
    const float u = x * x;
    float ps = fmaf(u, -2.5052108385e-8f, 2.7557319224e-6f);  // -1/11!, 1/9!
    ps = fmaf(u, ps, -1.9841269841e-4f);                        // -1/7!
    ps = fmaf(u, ps, 8.3333333333e-3f);                         // 1/5!
    ps = fmaf(u, ps, -1.6666666667e-1f);                        // -1/3!
    s = fmaf(x * u, ps, x);
    float pc = fmaf(u, 2.0876756988e-9f, -2.7557319224e-7f);    // 1/12!, -1/10!
    pc = fmaf(u, pc, 2.4801587302e-5f);                         // 1/8!
    pc = fmaf(u, pc, -1.3888888889e-3f);                        // -1/6!
    pc = fmaf(u, pc, 4.1666666667e-2f);                         // 1/4!
    pc = fmaf(u, pc, -0.5f);                                    // -1/2!
    c = fmaf(u, pc, 1.0f);
}

// sin and cos of a clamped theta from its FP64 pole distance, so that sin is
// relatively accurate next to either pole (the near-pole metric inverse).
__device__ __forceinline__ void pole_sincos(double th, float &s, float &c) {
    const bool south = th > 1.5707963267948966;
    const float d = (float)(south ? kPi - th : th);
    sincos_quadrant(d, s, c);
    c = south ? -c : c;
    s = fmaxf(s, 1.0e-7f);  // s^2 >= eps^2 as kerr.py:93
}

struct Deriv32 {
    float r, th, ph, pr, pth, H;
};

// Hamiltonian equations of kerr.py:285-303 written through
//   2 Sigma H = Delta p_r^2 + p_theta^2 + P^2 - W^2 / Delta,
//   P = p_phi / sin + a sin p_t,  W = (r^2 + a^2) p_t + a p_phi,
// which is g^{mu nu} p_mu p_nu of kerr.py:86-102 regrouped; x' = dH/dp and
// p' = -dH/dx are its exact derivatives (the quotient-rule sums of
// kerr.py:236-282 collapse to these few terms).
//
// Delta is evaluated as (r - r+)(r - r-) from the FP64 horizon distance
// r - r+: the expanded r^2 - 2r + a^2 cancels to nothing in FP32 within ~1e-7
// of the horizon, where 1/Delta then overflows (the horizon-proximity FP64
// island).
__device__ __forceinline__ void rhs32(double rd, double r_plus, float dpm, float s, float c, float pr, float pth,
                                      float pt, float pphi, float a, float a2, Deriv32 &d) {
    const float r = (float)rd;
    const float x = (float)(rd - r_plus);
    const float r2 = r * r;
    const float D = x * (x + dpm);
    const float Sg = fmaf(a2 * c, c, r2);
    const float iS = 1.0f / Sg;
    const float iD = 1.0f / D;
    const float is = 1.0f / s;
    const float W = fmaf(r2 + a2, pt, a * pphi);
    const float P = fmaf(a * s, pt, pphi * is);
    const float Q = W * iD;
    const float F = fmaf(D * pr, pr, fmaf(pth, pth, fmaf(P, P, -W * Q)));
    d.r = D * pr * iS;
    d.th = pth * iS;
    d.ph = fmaf(P, is, -a * Q) * iS;
    const float dFr = fmaf(2.0f * r - 2.0f, fmaf(pr, pr, Q * Q), -4.0f * r * pt * Q);
    d.pr = fmaf(-0.5f, dFr, F * r * iS) * iS;
    const float dFth = 2.0f * P * c * fmaf(a, pt, -pphi * is * is);
    d.pth = fmaf(-0.5f, dFth, -F * a2 * s * c * iS) * iS;
    d.H = 0.5f * F * iS;
}

struct Tracer32 {
    double r, th, ph;
    float pr, pth, pt, pphi, a, a2, dpm;
    float S0, S1, S2, S3, tau, drift, H0;
    float hs, hmin, hmax, L, max_tau;
    double r_cap, esc, r_plus;
    int steps, brick, max_steps;
    bool poison;
    int64_t out_idx;

    __device__ __forceinline__ void init(const ViewDev &v, int px, int py, int64_t out_index) {
        CameraRay c = camera_ray(v, px, py);
        r = v.r_obs;
        th = v.theta_obs;
        ph = v.phi_obs;
        pr = (float)c.pr;
        pth = (float)c.pth;
        pt = (float)c.pt;
        pphi = (float)c.pphi;
        a = (float)v.a;
        a2 = a * a;
        r_plus = v.r_plus;
        dpm = (float)(v.r_plus - v.r_minus);
        H0 = (float)c.H0;
        S0 = S1 = S2 = S3 = 0.0f;
        tau = 0.0f;
        drift = 0.0f;
        hs = (float)v.h_scale;
        hmin = (float)v.h_min;
        hmax = (float)v.h_max;
        L = (float)v.L;
        max_tau = (float)v.max_tau;
        r_cap = v.r_capture;
        esc = v.escape_radius;
        steps = 0;
        brick = 0;
        max_steps = v.max_steps;
        poison = false;
        out_idx = out_index;
    }

    // One RK2 geodesic step plus its brick segment.  Returns -1 while the ray
    // lives, else its BHN_RAY_* status.
    __device__ __forceinline__ int step(const Tables &T, const float4 *__restrict__ rec, int nt, int np) {
        const float rf = (float)r;
        const float h = fminf(fmaxf(hs * rf, hmin), hmax);
        float s, c;
        pole_sincos(th, s, c);
        Deriv32 k1;
        rhs32(r, r_plus, dpm, s, c, pr, pth, pt, pphi, a, a2, k1);
        drift = fmaxf(drift, fabsf(fabsf(k1.H) - H0));
        const float hh = 0.5f * h;
        const double rm = r + (double)(hh * k1.r);
        const double thm = safe_theta(th + (double)(hh * k1.th));
        pole_sincos(thm, s, c);
        Deriv32 k2;
        rhs32(rm, r_plus, dpm, s, c, fmaf(hh, k1.pr, pr), fmaf(hh, k1.pth, pth), pt, pphi, a, a2, k2);
        const float dr = h * k2.r, dph = h * k2.ph;
        const double rn = r + (double)dr;
        const double thn = safe_theta(th + (double)(h * k2.th));
        const double phn = ph + (double)dph;
        pr = fmaf(h, k2.pr, pr);
        pth = fmaf(h, k2.pth, pth);
        ++steps;
        const bool finite = isfinite(rn) && isfinite(thn) && isfinite(phn) && isfinite(pr) && isfinite(pth);

        // segment (y, y_n): accelerated_renderer.py:113-125
        if (tau < max_tau) {
            const double rmid = 0.5 * (r + rn), tmid = 0.5 * (th + thn), pmid = 0.5 * (ph + phn);
            const TableHeader &H = *T.h;
            if (!(rmid < T.gr[0] || rmid > T.gr[T.h->nr - 1]) && !(tmid < T.gt[0] || tmid > T.gt[nt - 1])) {
                ++brick;
                if (isnan(rmid) || isnan(tmid) || !isfinite(pmid)) {
                    poison = true;  // NaN coefficients in the reference -> nan_to_num -> 0
                } else {
                    const int nr = T.h->nr;
                    const int ir = locate_linear(T.gr, nr, rmid, H.kind_r, H.off_r, H.inv_r);
                    const int it = locate_linear(T.gt, nt, tmid, H.kind_t, H.off_t, H.inv_t);
                    const double pw = wrap_phi(pmid, T.gp[0]);
                    const int ip = locate_phi(T.gp, np, pw, H.kind_p, H.off_p, H.inv_p);
                    const int ip1 = ip + 1 == np ? 0 : ip + 1;
                    const float wr = (float)(rmid - T.gr[ir]) * T.idr[ir];
                    const float wt = (float)(tmid - T.gt[it]) * T.idt[it];
                    const float wp = (float)((pw >= T.gp[ip] ? pw : pw + kTwoPi) - T.gp[ip]) * T.idp[ip];
                    const float owr = 1.0f - wr, owt = 1.0f - wt, owp = 1.0f - wp;
                    const int64_t c00 = ((int64_t)ir * nt + it) * np;
                    const int64_t cells[4] = {c00, c00 + np, c00 + (int64_t)nt * np, c00 + (int64_t)nt * np + np};
                    const float wrt[4] = {owr * owt, owr * wt, wr * owt, wr * wt};
                    float cf[12];
#pragma unroll
                    for (int k = 0; k < 12; ++k) cf[k] = 0.0f;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 *p0 = rec + 3 * (cells[q] + ip);
                        const float4 *p1 = rec + 3 * (cells[q] + ip1);
                        const float w0 = wrt[q] * owp, w1 = wrt[q] * wp;
                        const float4 a0 = __ldg(p0), b0 = __ldg(p0 + 1), c0 = __ldg(p0 + 2);
                        const float4 a1 = __ldg(p1), b1 = __ldg(p1 + 1), c1 = __ldg(p1 + 2);
                        cf[0] = fmaf(w0, a0.x, fmaf(w1, a1.x, cf[0]));
                        cf[1] = fmaf(w0, a0.y, fmaf(w1, a1.y, cf[1]));
                        cf[2] = fmaf(w0, a0.z, fmaf(w1, a1.z, cf[2]));
                        cf[3] = fmaf(w0, a0.w, fmaf(w1, a1.w, cf[3]));
                        cf[4] = fmaf(w0, b0.x, fmaf(w1, b1.x, cf[4]));
                        cf[5] = fmaf(w0, b0.y, fmaf(w1, b1.y, cf[5]));
                        cf[6] = fmaf(w0, b0.z, fmaf(w1, b1.z, cf[6]));
                        cf[7] = fmaf(w0, b0.w, fmaf(w1, b1.w, cf[7]));
                        cf[8] = fmaf(w0, c0.x, fmaf(w1, c1.x, cf[8]));
                        cf[9] = fmaf(w0, c0.y, fmaf(w1, c1.y, cf[9]));
                        cf[10] = fmaf(w0, c0.z, fmaf(w1, c1.z, cf[10]));
                    }
                    // ds = L * max(|d(r, theta, phi)|, 1e-14) (accelerated_renderer.py:120-121)
                    const float dth = (float)(thn - th);
                    const float len = sqrtf(fmaf(dr, dr, fmaf(dth, dth, dph * dph)));
                    const float ds = L * fmaxf(len, 1.0e-14f);
                    // Stokes RK2 (lib.rs:210-225) with K of native_kernels.py:213-222
                    const float j0 = cf[0], j1 = cf[1], j2 = cf[2], j3 = cf[3];
                    const float ai = cf[4], aq = cf[5], au = cf[6], av = cf[7];
                    const float rv = cf[8], rq = cf[9], ru = cf[10];
                    float k0 = j0 - (ai * S0 + aq * S1 + au * S2 + av * S3);
                    float k1q = j1 - (aq * S0 + ai * S1 + rv * S2 - ru * S3);
                    float k2u = j2 - (au * S0 - rv * S1 + ai * S2 + rq * S3);
                    float k3v = j3 - (av * S0 + ru * S1 - rq * S2 + ai * S3);
                    const float hd = 0.5f * ds;
                    const float m0 = fmaf(hd, k0, S0), m1 = fmaf(hd, k1q, S1), m2 = fmaf(hd, k2u, S2),
                                m3 = fmaf(hd, k3v, S3);
                    k0 = j0 - (ai * m0 + aq * m1 + au * m2 + av * m3);
                    k1q = j1 - (aq * m0 + ai * m1 + rv * m2 - ru * m3);
                    k2u = j2 - (au * m0 - rv * m1 + ai * m2 + rq * m3);
                    k3v = j3 - (av * m0 + ru * m1 - rq * m2 + ai * m3);
                    S0 = fmaf(ds, k0, S0);
                    S1 = fmaf(ds, k1q, S1);
                    S2 = fmaf(ds, k2u, S2);
                    S3 = fmaf(ds, k3v, S3);
                    tau = fmaf(fmaxf(ai, 0.0f), ds, tau);
                }
            }
        }
        const double r_old = r;
        r = rn;
        th = thn;
        ph = phn;
        // kerr.py:364-377, in FP64
        if (!finite) return BHN_RAY_INVALID;
        if (tau >= max_tau) return BHN_RAY_OPAQUE;
        if (rn <= r_cap) return BHN_RAY_CAPTURED;
        if (rn > esc && rn > r_old) return BHN_RAY_ESCAPED;
        if (steps >= max_steps) return BHN_RAY_MAX_STEPS;
        return -1;
    }

    __device__ __forceinline__ void finish(void *out, int status) {
        // drift at the final state (kerr.py:360, 367)
        if (status != BHN_RAY_INVALID) {
            float s, c;
            pole_sincos(th, s, c);
            Deriv32 k;
            rhs32(r, r_plus, dpm, s, c, pr, pth, pt, pphi, a, a2, k);
            drift = fmaxf(drift, fabsf(fabsf(k.H) - H0));
        }
        float4 o;
        // np.nan_to_num(S, nan=0, posinf=0, neginf=0) (accelerated_renderer.py:126)
        o.x = (poison || !isfinite(S0)) ? 0.0f : S0;
        o.y = (poison || !isfinite(S1)) ? 0.0f : S1;
        o.z = (poison || !isfinite(S2)) ? 0.0f : S2;
        o.w = (poison || !isfinite(S3)) ? 0.0f : S3;
        reinterpret_cast<float4 *>(out)[out_idx] = o;
    }

    static __device__ __forceinline__ void write_zero(void *out, int64_t idx) {
        reinterpret_cast<float4 *>(out)[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
};

// ------------------------------------------------------------ FP64 tracer
// kerr.py:52-64, :86-102, :236-303 in FP64 (the oracle's formulation).
struct Metric64 {
    double g00, g03, g11, g22, g33;
};
__device__ __forceinline__ void metric_con64(double r, double th, double a, Metric64 &g, double &sig, double &dlt,
                                             double &A, double &s, double &c) {
    s = sin(th);
    c = cos(th);
    sig = r * r + a * a * (c * c);
    dlt = r * r - 2.0 * r + a * a;
    A = (r * r + a * a) * (r * r + a * a) - a * a * dlt * (s * s);
    const double s2 = fmax(s * s, kEpsTheta * kEpsTheta);
    g.g00 = -A / (sig * dlt);
    g.g03 = -2.0 * a * r / (sig * dlt);
    g.g11 = dlt / sig;
    g.g22 = 1.0 / sig;
    g.g33 = (dlt - a * a * s2) / (sig * dlt * s2);
}

__device__ __forceinline__ void metric_deriv64(double r, double a, double s, double c, double sig, double dlt,
                                               double A, bool wrt_theta, Metric64 &o) {
    const double s2 = fmax(s * s, kEpsTheta * kEpsTheta);
    const double ds2 = 2.0 * s * c;
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
    double den = sig * dlt;
    double den_p = sig_p * dlt + sig * dlt_p;
    o.g00 = -((A_p * den - A * den_p) / (den * den));
    const double num = -2.0 * a * r;
    const double num_p = !wrt_theta ? -2.0 * a : 0.0;
    o.g03 = (num_p * den - num * den_p) / (den * den);
    o.g11 = (dlt_p * sig - dlt * sig_p) / (sig * sig);
    o.g22 = -sig_p / (sig * sig);
    const double num2 = dlt - a * a * s2;
    const double num2_p = dlt_p - a * a * s2_p;
    den = sig * dlt * s2;
    den_p = sig_p * dlt * s2 + sig * dlt_p * s2 + sig * dlt * s2_p;
    o.g33 = (num2_p * den - num2 * den_p) / (den * den);
}

struct Deriv64 {
    double r, th, ph, pr, pth, H;
};

__device__ __forceinline__ double quad64(const Metric64 &m, double pt, double pr, double pth, double pphi) {
    return m.g00 * pt * pt + 2.0 * m.g03 * pt * pphi + m.g11 * pr * pr + m.g22 * pth * pth + m.g33 * pphi * pphi;
}

__device__ __forceinline__ void rhs64(double r, double th_in, double pr, double pth, double pt, double pphi, double a,
                                      Deriv64 &d) {
    const double th = safe_theta(th_in);
    Metric64 g, gr, gth;
    double sig, dlt, A, s, c;
    metric_con64(r, th, a, g, sig, dlt, A, s, c);
    d.r = g.g11 * pr;
    d.th = g.g22 * pth;
    d.ph = g.g03 * pt + g.g33 * pphi;
    metric_deriv64(r, a, s, c, sig, dlt, A, false, gr);
    metric_deriv64(r, a, s, c, sig, dlt, A, true, gth);
    d.pr = -0.5 * quad64(gr, pt, pr, pth, pphi);
    d.pth = -0.5 * quad64(gth, pt, pr, pth, pphi);
    d.H = 0.5 * quad64(g, pt, pr, pth, pphi);
}

struct Tracer64 {
    double r, th, ph, pr, pth, pt, pphi, a;
    double S0, S1, S2, S3, tau, drift, H0;
    double hs, hmin, hmax, L, max_tau, r_cap, esc;
    int steps, brick, max_steps;
    bool poison;
    int64_t out_idx;

    __device__ __forceinline__ void init(const ViewDev &v, int px, int py, int64_t out_index) {
        CameraRay c = camera_ray(v, px, py);
        r = v.r_obs;
        th = v.theta_obs;
        ph = v.phi_obs;
        pr = c.pr;
        pth = c.pth;
        pt = c.pt;
        pphi = c.pphi;
        a = v.a;
        H0 = c.H0;
        S0 = S1 = S2 = S3 = 0.0;
        tau = 0.0;
        drift = 0.0;
        hs = v.h_scale;
        hmin = v.h_min;
        hmax = v.h_max;
        L = v.L;
        max_tau = v.max_tau;
        r_cap = v.r_capture;
        esc = v.escape_radius;
        steps = 0;
        brick = 0;
        max_steps = v.max_steps;
        poison = false;
        out_idx = out_index;
    }

    __device__ __forceinline__ int step(const Tables &T, const double2 *__restrict__ rec, int nt, int np) {
        const double h = fmin(fmax(hs * r, hmin), hmax);
        Deriv64 k1, k2;
        rhs64(r, th, pr, pth, pt, pphi, a, k1);
        drift = fmax(drift, fabs(fabs(k1.H) - H0));
        const double hh = 0.5 * h;
        rhs64(r + hh * k1.r, th + hh * k1.th, pr + hh * k1.pr, pth + hh * k1.pth, pt, pphi, a, k2);
        const double rn = r + h * k2.r;
        const double thn = safe_theta(th + h * k2.th);
        const double phn = ph + h * k2.ph;
        pr = pr + h * k2.pr;
        pth = pth + h * k2.pth;
        ++steps;
        const bool finite = isfinite(rn) && isfinite(thn) && isfinite(phn) && isfinite(pr) && isfinite(pth);
        if (tau < max_tau) {
            const double rmid = 0.5 * (r + rn), tmid = 0.5 * (th + thn), pmid = 0.5 * (ph + phn);
            const TableHeader &H = *T.h;
            const int nr = H.nr;
            if (!(rmid < T.gr[0] || rmid > T.gr[nr - 1]) && !(tmid < T.gt[0] || tmid > T.gt[nt - 1])) {
                ++brick;
                if (isnan(rmid) || isnan(tmid) || !isfinite(pmid)) {
                    poison = true;
                } else {
                    const int ir = locate_linear(T.gr, nr, rmid, H.kind_r, H.off_r, H.inv_r);
                    const int it = locate_linear(T.gt, nt, tmid, H.kind_t, H.off_t, H.inv_t);
                    const double pw = wrap_phi(pmid, T.gp[0]);
                    const int ip = locate_phi(T.gp, np, pw, H.kind_p, H.off_p, H.inv_p);
                    const int ip1 = ip + 1 == np ? 0 : ip + 1;
                    // native_kernels.py:145 / :158-160 weights in FP64
                    const double wr = (rmid - T.gr[ir]) / (T.gr[ir + 1] - T.gr[ir]);
                    const double wt = (tmid - T.gt[it]) / (T.gt[it + 1] - T.gt[it]);
                    const double hi = ip1 > ip ? T.gp[ip1] : T.gp[0] + kTwoPi;
                    const double pp = pw >= T.gp[ip] ? pw : pw + kTwoPi;
                    const double wp = (pp - T.gp[ip]) / (hi - T.gp[ip]);
                    const int64_t c00 = ((int64_t)ir * nt + it) * np;
                    const int64_t cr0t0 = c00, cr0t1 = c00 + np, cr1t0 = c00 + (int64_t)nt * np,
                                  cr1t1 = cr1t0 + np;
                    double cf[12];
                    // native_kernels.py:180-186: phi lerps, then theta, then r
#pragma unroll
                    for (int k2i = 0; k2i < 6; ++k2i) {
                        const double2 v000 = rec[6 * (cr0t0 + ip) + k2i], v001 = rec[6 * (cr0t0 + ip1) + k2i];
                        const double2 v010 = rec[6 * (cr0t1 + ip) + k2i], v011 = rec[6 * (cr0t1 + ip1) + k2i];
                        const double2 v100 = rec[6 * (cr1t0 + ip) + k2i], v101 = rec[6 * (cr1t0 + ip1) + k2i];
                        const double2 v110 = rec[6 * (cr1t1 + ip) + k2i], v111 = rec[6 * (cr1t1 + ip1) + k2i];
                        double c00x = (1.0 - wp) * v000.x + wp * v001.x, c00y = (1.0 - wp) * v000.y + wp * v001.y;
                        double c01x = (1.0 - wp) * v010.x + wp * v011.x, c01y = (1.0 - wp) * v010.y + wp * v011.y;
                        double c10x = (1.0 - wp) * v100.x + wp * v101.x, c10y = (1.0 - wp) * v100.y + wp * v101.y;
                        double c11x = (1.0 - wp) * v110.x + wp * v111.x, c11y = (1.0 - wp) * v110.y + wp * v111.y;
                        double c0x = (1.0 - wt) * c00x + wt * c01x, c0y = (1.0 - wt) * c00y + wt * c01y;
                        double c1x = (1.0 - wt) * c10x + wt * c11x, c1y = (1.0 - wt) * c10y + wt * c11y;
                        cf[2 * k2i] = (1.0 - wr) * c0x + wr * c1x;
                        cf[2 * k2i + 1] = (1.0 - wr) * c0y + wr * c1y;
                    }
                    const double d0 = rn - r, d1 = thn - th, d2 = phn - ph;
                    double dl = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                    if (1.0e-14 > dl) dl = 1.0e-14;
                    double ds = L * dl;
                    if (ds < 0.0) ds = 0.0;
                    const double j0 = cf[0], j1 = cf[1], j2 = cf[2], j3 = cf[3];
                    const double ai = cf[4], aq = cf[5], au = cf[6], av = cf[7];
                    const double rv = cf[8], rq = cf[9], ru = cf[10];
                    double k0 = j0 - (ai * S0 + aq * S1 + au * S2 + av * S3);
                    double kq = j1 - (aq * S0 + ai * S1 + rv * S2 - ru * S3);
                    double ku = j2 - (au * S0 - rv * S1 + ai * S2 + rq * S3);
                    double kv = j3 - (av * S0 + ru * S1 - rq * S2 + ai * S3);
                    const double hd = 0.5 * ds;
                    const double m0 = S0 + hd * k0, m1 = S1 + hd * kq, m2 = S2 + hd * ku, m3 = S3 + hd * kv;
                    k0 = j0 - (ai * m0 + aq * m1 + au * m2 + av * m3);
                    kq = j1 - (aq * m0 + ai * m1 + rv * m2 - ru * m3);
                    ku = j2 - (au * m0 - rv * m1 + ai * m2 + rq * m3);
                    kv = j3 - (av * m0 + ru * m1 - rq * m2 + ai * m3);
                    S0 = S0 + ds * k0;
                    S1 = S1 + ds * kq;
                    S2 = S2 + ds * ku;
                    S3 = S3 + ds * kv;
                    tau += (0.0 > ai ? 0.0 : ai) * ds;
                }
            }
        }
        const double r_old = r;
        r = rn;
        th = thn;
        ph = phn;
        if (!finite) return BHN_RAY_INVALID;
        if (tau >= max_tau) return BHN_RAY_OPAQUE;
        if (rn <= r_cap) return BHN_RAY_CAPTURED;
        if (rn > esc && rn > r_old) return BHN_RAY_ESCAPED;
        if (steps >= max_steps) return BHN_RAY_MAX_STEPS;
        return -1;
    }

    __device__ __forceinline__ void finish(void *out, int status) {
        if (status != BHN_RAY_INVALID) {
            Deriv64 k;
            rhs64(r, th, pr, pth, pt, pphi, a, k);
            drift = fmax(drift, fabs(fabs(k.H) - H0));
        }
        double2 *o = reinterpret_cast<double2 *>(out) + 2 * out_idx;
        o[0] = make_double2((poison || !isfinite(S0)) ? 0.0 : S0, (poison || !isfinite(S1)) ? 0.0 : S1);
        o[1] = make_double2((poison || !isfinite(S2)) ? 0.0 : S2, (poison || !isfinite(S3)) ? 0.0 : S3);
    }

    static __device__ __forceinline__ void write_zero(void *out, int64_t idx) {
        double2 *o = reinterpret_cast<double2 *>(out) + 2 * idx;
        o[0] = make_double2(0.0, 0.0);
        o[1] = make_double2(0.0, 0.0);
    }
};

template <class T> struct RecordOf;
template <> struct RecordOf<Tracer32> { using type = float4; };
template <> struct RecordOf<Tracer64> { using type = double2; };

// ------------------------------------------------------------ persistent loop
template <class Tracer>
__global__ void __launch_bounds__(256) render_kernel(const RenderParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    // grid tables and the view prefix live in shared memory for the whole launch
    {
        const int4 *src = reinterpret_cast<const int4 *>(P.tables);
        int4 *dst = reinterpret_cast<int4 *>(smem);
        for (int i = threadIdx.x; i < P.tables_bytes / 16; i += blockDim.x) dst[i] = src[i];
        int64_t *vb = reinterpret_cast<int64_t *>(smem + P.tables_bytes);
        for (int i = threadIdx.x; i <= P.n_views; i += blockDim.x) vb[i] = P.ray_begin[i];
    }
    __syncthreads();
    const Tables T = tables_at(smem, P.nr, P.nt, P.np);
    const int64_t *vbegin = reinterpret_cast<const int64_t *>(smem + P.tables_bytes);
    const unsigned long long total = vbegin[P.n_views];
    using Rec = typename RecordOf<Tracer>::type;
    const Rec *rec = reinterpret_cast<const Rec *>(P.records);

    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    Tracer tr;
    bool alive = false, exhausted = false;
    LaneCounters cnt;
    cnt.steps = cnt.brick = 0;
    cnt.rays = 0;
    for (int k = 0; k < 5; ++k) cnt.status[k] = 0;
    cnt.max_drift = 0.0f;
    cnt.max_drift_escaped = 0.0f;
    unsigned long long fetches = 0;

    while (true) {
        const unsigned dead = __ballot_sync(kFull, !alive);
        const int ndead = __popc(dead);
        if (!exhausted && ndead > 0 && (ndead >= P.refill_min || ndead == 32)) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(&P.q->next, (unsigned long long)ndead);
            base = __shfl_sync(kFull, base, 0);
            ++fetches;
            if (base + (unsigned long long)ndead >= total) exhausted = true;
            if (!alive) {
                const unsigned long long slot = base + __popc(dead & lt_mask);
                if (slot < total) {
                    const int vi = P.n_views == 1 ? 0 : find_view(vbegin, P.n_views, (int64_t)slot);
                    const ViewDev &v = P.views[vi];
                    const PixelRef px = pixel_of(v, (int64_t)slot - vbegin[vi], P.tile_w, P.tile_h);
                    if (v.valid && v.max_steps > 0) {
                        tr.init(v, px.px, px.py, px.out_idx);
                        alive = true;
                    } else {
                        // no step is taken: the reference returns a zero Stokes vector
                        Tracer::write_zero(P.out, px.out_idx);
                        cnt.rays += 1;
                        const int zst = v.valid ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID;
#pragma unroll
                        for (int k = 0; k < 5; ++k) cnt.status[k] += (zst == k);
                        if (P.ray_steps) P.ray_steps[px.out_idx] = 0;
                        if (P.ray_status) P.ray_status[px.out_idx] = (uint8_t)(v.valid ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID);
                        if (P.ray_drift) P.ray_drift[px.out_idx] = 0.0f;
                    }
                }
            }
        }
        if (__ballot_sync(kFull, alive) == 0) {
            if (exhausted) break;
            continue;
        }
        if (alive) {
            const int st = tr.step(T, rec, P.nt, P.np);
            if (st >= 0) {
                tr.finish(P.out, st);
                cnt.steps += (unsigned long long)tr.steps;
                cnt.brick += (unsigned long long)tr.brick;
                cnt.rays += 1;
#pragma unroll
                for (int k = 0; k < 5; ++k) cnt.status[k] += (st == k);
                cnt.max_drift = fmaxf(cnt.max_drift, (float)tr.drift);
                if (st == BHN_RAY_ESCAPED) cnt.max_drift_escaped = fmaxf(cnt.max_drift_escaped, (float)tr.drift);
                if (P.ray_steps) P.ray_steps[tr.out_idx] = tr.steps;
                if (P.ray_status) P.ray_status[tr.out_idx] = (uint8_t)st;
                if (P.ray_drift) P.ray_drift[tr.out_idx] = (float)tr.drift;
                alive = false;
            }
        }
    }

    // launch totals: warp reduction, one atomic per warp and counter
    for (int o = 16; o > 0; o >>= 1) {
        cnt.steps += __shfl_down_sync(kFull, cnt.steps, o);
        cnt.brick += __shfl_down_sync(kFull, cnt.brick, o);
        cnt.rays += __shfl_down_sync(kFull, cnt.rays, o);
#pragma unroll
        for (int k = 0; k < 5; ++k) cnt.status[k] += __shfl_down_sync(kFull, cnt.status[k], o);
        cnt.max_drift = fmaxf(cnt.max_drift, __shfl_down_sync(kFull, cnt.max_drift, o));
        cnt.max_drift_escaped = fmaxf(cnt.max_drift_escaped, __shfl_down_sync(kFull, cnt.max_drift_escaped, o));
    }
    if (lane == 0 && P.stats) {
        atomicAdd(&P.stats->ray_steps, cnt.steps);
        atomicAdd(&P.stats->brick_steps, cnt.brick);
        atomicAdd(&P.stats->rays, (unsigned long long)cnt.rays);
        for (int k = 0; k < 5; ++k)
            if (cnt.status[k]) atomicAdd(&P.stats->status[k], (unsigned long long)cnt.status[k]);
        atomicAdd(&P.stats->queue_fetches, fetches);
        // non-negative floats order like their bit patterns
        atomicMax(reinterpret_cast<unsigned int *>(&P.stats->max_h_drift), __float_as_uint(cnt.max_drift));
        atomicMax(reinterpret_cast<unsigned int *>(&P.stats->max_h_drift_escaped),
                  __float_as_uint(cnt.max_drift_escaped));
    }
}

static int check_config(const bhn_render_config *cfg) {
    if (!cfg) return fail(BHN_ERR_VALUE, "render config must not be NULL");
    if (cfg->block_threads < 32 || cfg->block_threads > 256 || cfg->block_threads % 32)
        return fail(BHN_ERR_VALUE, "block_threads must be a multiple of 32 in [32, 256]");
    if (cfg->blocks_per_sm < 1 || cfg->blocks_per_sm > 32) return fail(BHN_ERR_VALUE, "blocks_per_sm must be in [1, 32]");
    if (cfg->tile_w < 1 || cfg->tile_h < 1 || cfg->tile_w * cfg->tile_h > 4096)
        return fail(BHN_ERR_VALUE, "tile_w * tile_h must be in [1, 4096]");
    if (cfg->refill_min < 1 || cfg->refill_min > 32) return fail(BHN_ERR_VALUE, "refill_min must be in [1, 32]");
    if (cfg->precision != 0 && cfg->precision != 1) return fail(BHN_ERR_VALUE, "precision must be 0 (fp32) or 1 (fp64)");
    return BHN_OK;
}

static int launch_render(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                         const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                         int64_t scratch_bytes, bhn_render_stats *stats, cudaStream_t s) {
    int rc = check_config(cfg);
    if (rc) return rc;
    if (n_views < 1) return fail(BHN_ERR_VALUE, "at least one view is required");
    if (!records || !tables || !out || !scratch) return fail(BHN_ERR_VALUE, "records, tables, out and scratch must not be NULL");
    if (nr < 2 || nt < 2 || np < 2) return fail(BHN_ERR_VALUE, "brick grids must contain at least 2 values");
    ScratchLayout L = scratch_layout(n_views);
    if (scratch_bytes < L.total) return fail(BHN_ERR_VALUE, "scratch buffer is smaller than bhn_render_scratch_bytes()");
    if (reinterpret_cast<uintptr_t>(records) % 16 || reinterpret_cast<uintptr_t>(tables) % 16 ||
        reinterpret_cast<uintptr_t>(scratch) % 256 || reinterpret_cast<uintptr_t>(out) % 16)
        return fail(BHN_ERR_VALUE, "records/tables/out must be 16-byte and scratch 256-byte aligned");
    const int tables_bytes = (int)table_layout(nr, nt, np).total;
    const int smem = tables_bytes + 8 * (n_views + 1);
    if (smem > 200 * 1024) return fail(BHN_ERR_VALUE, "brick grids plus views exceed the shared-memory table budget");
    char *sc = static_cast<char *>(scratch);
    RenderParams P;
    P.records = records;
    P.tables = tables;
    P.nr = nr;
    P.nt = nt;
    P.np = np;
    P.n_views = n_views;
    P.views = reinterpret_cast<const ViewDev *>(sc + L.views);
    P.ray_begin = reinterpret_cast<const int64_t *>(sc + L.ray_begin);
    P.q = reinterpret_cast<QueueState *>(sc + L.queue);
    P.stats = stats ? stats : reinterpret_cast<bhn_render_stats *>(sc + L.stats);
    P.out = out;
    P.ray_steps = ray_out ? ray_out->steps : nullptr;
    P.ray_status = ray_out ? ray_out->status : nullptr;
    P.ray_drift = ray_out ? ray_out->h_drift : nullptr;
    P.tile_w = cfg->tile_w;
    P.tile_h = cfg->tile_h;
    P.refill_min = cfg->refill_min;
    P.tables_bytes = tables_bytes;
    const int sms = sm_count_current_device();
    if (sms <= 0) return fail(BHN_ERR_CUDA, "cannot query the SM count");
    const dim3 grid((unsigned)(sms * cfg->blocks_per_sm)), block((unsigned)cfg->block_threads);
    BHN_CUDA_TRY(cudaMemsetAsync(&P.q->next, 0, sizeof(unsigned long long), s));
    BHN_CUDA_TRY(cudaMemsetAsync(P.stats, 0, sizeof(bhn_render_stats), s));
    if (cfg->precision == 0) {
        if (smem > 48 * 1024)
            BHN_CUDA_TRY(cudaFuncSetAttribute(render_kernel<Tracer32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        render_kernel<Tracer32><<<grid, block, smem, s>>>(P);
    } else {
        if (smem > 48 * 1024)
            BHN_CUDA_TRY(cudaFuncSetAttribute(render_kernel<Tracer64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        render_kernel<Tracer64><<<grid, block, smem, s>>>(P);
    }
    BHN_LAUNCH_CHECK("render_kernel");
    return BHN_OK;
}

}  // namespace bhn

using namespace bhn;

struct bhn_graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

extern "C" {

int64_t bhn_render_scratch_bytes(int32_t n_views) {
    if (n_views < 1) return 0;
    return scratch_layout(n_views).total;
}

int bhn_render_prepare(const bhn_view *h_views, int32_t n_views, void *scratch, int64_t scratch_bytes, void *stream) {
    if (!h_views || n_views < 1) return fail(BHN_ERR_VALUE, "at least one view is required");
    if (n_views > (1 << 20)) return fail(BHN_ERR_VALUE, "too many views");
    ScratchLayout L = scratch_layout(n_views);
    if (!scratch || scratch_bytes < L.total) return fail(BHN_ERR_VALUE, "scratch buffer is smaller than bhn_render_scratch_bytes()");
    if (reinterpret_cast<uintptr_t>(scratch) % 256) return fail(BHN_ERR_VALUE, "scratch must be 256-byte aligned");
    for (int i = 0; i < n_views; ++i) {
        const bhn_view &v = h_views[i];
        if (v.width < 1 || v.height < 1 || v.crop_w < 1 || v.crop_h < 1 || v.x0 < 0 || v.y0 < 0 ||
            v.x0 + v.crop_w > v.width || v.y0 + v.crop_h > v.height)
            return fail(BHN_ERR_VALUE, "view crop rectangle must lie inside the image");
        if ((int64_t)v.crop_w * v.crop_h > (int64_t)1 << 30) return fail(BHN_ERR_VALUE, "view has too many pixels");
        if (v.max_steps < 0) return fail(BHN_ERR_VALUE, "max_steps must be non-negative");
        if (!(std::isfinite(v.spin_a) && std::fabs(v.spin_a) < 1.0))
            return fail(BHN_ERR_VALUE, "Kerr spin must be finite and satisfy |a| < 1 for this integrator");
        if (!(v.h_min > 0.0 && v.h_max >= v.h_min && std::isfinite(v.h_max) && std::isfinite(v.h_scale)))
            return fail(BHN_ERR_VALUE, "step bounds must satisfy 0 < h_min <= h_max");
        if (v.out_offset < 0) return fail(BHN_ERR_VALUE, "out_offset must be non-negative");
    }
    cudaStream_t s = as_stream(stream);
    char *sc = static_cast<char *>(scratch);
    BHN_CUDA_TRY(cudaMemcpyAsync(sc + L.raw_views, h_views, sizeof(bhn_view) * n_views, cudaMemcpyHostToDevice, s));
    setup_views_kernel<<<1, 256, 0, s>>>(reinterpret_cast<const bhn_view *>(sc + L.raw_views), n_views,
                                         reinterpret_cast<ViewDev *>(sc + L.views),
                                         reinterpret_cast<int64_t *>(sc + L.ray_begin),
                                         reinterpret_cast<QueueState *>(sc + L.queue));
    BHN_LAUNCH_CHECK("setup_views_kernel");
    return BHN_OK;
}

int bhn_render_launch(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                      const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                      int64_t scratch_bytes, bhn_render_stats *stats, void *stream) {
    return launch_render(records, tables, nr, nt, np, n_views, cfg, out, ray_out, scratch, scratch_bytes, stats,
                         as_stream(stream));
}

int bhn_graph_create(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                     const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                     int64_t scratch_bytes, bhn_render_stats *stats, bhn_graph **graph) {
    if (!graph) return fail(BHN_ERR_VALUE, "graph must not be NULL");
    *graph = nullptr;
    cudaStream_t cs;
    BHN_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return cuda_fail(e, "cudaStreamBeginCapture");
    }
    int rc = launch_render(records, tables, nr, nt, np, n_views, cfg, out, ray_out, scratch, scratch_bytes, stats, cs);
    e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc != BHN_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    *graph = new bhn_graph{g, ex};
    return BHN_OK;
}

int bhn_graph_launch(bhn_graph *graph, void *stream) {
    if (!graph) return fail(BHN_ERR_VALUE, "graph must not be NULL");
    BHN_CUDA_TRY(cudaGraphLaunch(graph->exec, as_stream(stream)));
    return BHN_OK;
}

int bhn_graph_destroy(bhn_graph *graph) {
    if (!graph) return BHN_OK;
    cudaGraphExecDestroy(graph->exec);
    cudaGraphDestroy(graph->graph);
    delete graph;
    return BHN_OK;
}

}  // extern "C"
