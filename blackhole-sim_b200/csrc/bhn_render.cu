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
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>

#include "bhn_internal.cuh"

namespace bhn {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------ view set-up
__device__ __forceinline__ double safe_theta(double th) {  // kerr.py:35-36
    return fmin(fmax(th, kEpsTheta), kPi - kEpsTheta);
}

// Rays with small axial angular momentum |p_phi| run first.  Only they can
// come close to the spin axis, where the clamped sin(theta) (kerr.py:93)
// shrinks the useful step and such rays run up to max_steps -- several times
// longer than the rest; a persistent launch would otherwise finish with these
// few rays alone on the GPU.  For a camera without roll, p_phi of a ray is
// sqrt(g_phiphi) n_phi with n_phi = ndc_x tan_x / |n| (the ZAMO part cancels:
// g_tphi + g_phiphi omega = 0), so |p_phi| < kAxisBandPphi is a band of image
// columns; the order inside and outside the band stays the tile order.  It
// changes which ray a warp takes when, never a ray's result.
constexpr double kAxisBandPphi = 0.5;

__global__ void setup_views_kernel(const bhn_view *__restrict__ raw, int n, ViewDev *__restrict__ views,
                                   int64_t *__restrict__ ray_begin, int64_t *__restrict__ axis_begin, QueueState *q) {
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
        // prograde equatorial circular photon orbit, r = 2 (1 + cos(2/3 arccos(-|a|))) (Bardeen, Press &
        // Teukolsky 1972): the innermost spherical photon orbit, inside which an inbound ray cannot turn
        d.r_photon = 2.0 * (1.0 + cos((2.0 / 3.0) * acos(-fabs(a))));
        d.flags = v.flags;
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
        // |ndc_x| < u  =>  |p_phi| <= sqrt(g_phiphi) |ndc_x| tan_x < kAxisBandPphi (|n| >= 1)
        d.axis_x0 = d.axis_x1 = 0;
        if (d.valid && !d.has_roll && d.crop_w > 0 && d.crop_h > 0) {
            const double u = kAxisBandPphi / (sqrt(d.gcov33) * d.tan_x);
            const double lo = fmax((1.0 - u) * 0.5 * d.width_d - 0.5, -1.0);
            const double hi = fmin((1.0 + u) * 0.5 * d.width_d - 0.5, d.width_d);
            const int c0 = (int)ceil(lo) - v.x0, c1 = (int)floor(hi) + 1 - v.x0;
            d.axis_x0 = max(0, min(c0, v.crop_w));
            d.axis_x1 = max(d.axis_x0, min(c1, v.crop_w));
        }
        views[i] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t acc = 0, acc_axis = 0;
        for (int i = 0; i < n; ++i) {
            views[i].ray_begin = acc;
            views[i].axis_begin = acc_axis;
            ray_begin[i] = acc;
            axis_begin[i] = acc_axis;
            acc += views[i].ray_count;
            acc_axis += (int64_t)(views[i].axis_x1 - views[i].axis_x0) * views[i].crop_h;
        }
        ray_begin[n] = acc;
        axis_begin[n] = acc_axis;
        q->total = (unsigned long long)acc;
        q->n_views = (uint32_t)n;
        q->error_flags = 0;  // bit 0: the brick renderer's two-warp form gave up a wait
    }
}

// ------------------------------------------------------------ shared pieces
struct PixelRef {
    int32_t px, py;      // absolute pixel
    int64_t out_idx;     // index into the output image buffer
};

// Ray k of the crop columns [cx0, cx0 + cw) of a view (all crop rows) in tile
// order: bands of tile_h rows, tiles of tile_w columns inside a band (the last
// band / tile of a band may be narrower).
__device__ __forceinline__ PixelRef pixel_in_columns(const ViewDev &v, int64_t k, int cx0, int cw, int tw, int th) {
    const int ch = v.crop_h;
    const int kk = (int)k;
    const int band_rays = th * cw;
    const int band = kk / band_rays;
    const int kb = kk - band * band_rays;
    const int bh = min(th, ch - band * th);
    const int tile = kb / (tw * bh);
    const int kt = kb - tile * tw * bh;
    const int tw_eff = min(tw, cw - tile * tw);
    const int lx = cx0 + tile * tw + kt % tw_eff;
    const int ly = band * th + kt / tw_eff;
    PixelRef p;
    p.px = v.x0 + lx;
    p.py = v.y0 + ly;
    p.out_idx = v.out_offset + (int64_t)ly * v.crop_w + lx;
    return p;
}

// Ray k of a view's crop in tile order.
__device__ __forceinline__ PixelRef pixel_of(const ViewDev &v, int64_t k, int tw, int th) {
    return pixel_in_columns(v, k, 0, v.crop_w, tw, th);
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

// Per-view constants of the step loop, staged in shared memory (one entry per
// view; a lane keeps only its view index in registers).
struct __align__(16) StepConst {
    float a, a2, dpm, hs;               // spin, spin^2, r+ - r-, step scale
    float hmin, hmax, L, max_tau;
    float rp_h, rp_l, rcap_h, rcap_l;   // r+ and the capture radius as float pairs (value = hi + lo)
    float esc, r_guard, r_near, pad;    // escape radius, horizon-guard radius (0 = off), FP64-island radius
    int max_steps, pad1, pad2, pad3;
};

// Launch totals of one block, in shared memory (updated once per finished ray).
struct BlockCounters {
    unsigned long long steps, brick, fetches;
    unsigned int rays, status[5];
    float max_drift, max_drift_escaped;
};

struct RenderParams {
    const void *records;
    const void *tables;
    int nr, nt, np, n_views;
    const ViewDev *views;
    const int64_t *ray_begin;
    const int64_t *axis_begin;  // prefix of the views' axis-band rays
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

// Largest i with ray_begin[i] - axis_begin[i] <= slot (the views' rays outside
// their axis bands, view after view).
__device__ __forceinline__ int find_view_rest(const int64_t *ray_begin, const int64_t *axis_begin, int n,
                                              int64_t slot) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (ray_begin[mid] - axis_begin[mid] <= slot) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Queue slot -> (view, pixel) of the render kernel: first the axis-band rays of
// every view, then every view's remaining rays (left of the band, then right).
__device__ __forceinline__ PixelRef ordered_pixel(const ViewDev *views, const int64_t *ray_begin,
                                                  const int64_t *axis_begin, int n, int64_t slot, int tw, int th,
                                                  int &vi) {
    const int64_t n_axis = axis_begin[n];
    if (slot < n_axis) {
        vi = n == 1 ? 0 : find_view(axis_begin, n, slot);
        const ViewDev &v = views[vi];
        return pixel_in_columns(v, slot - axis_begin[vi], v.axis_x0, v.axis_x1 - v.axis_x0, tw, th);
    }
    const int64_t s = slot - n_axis;
    vi = n == 1 ? 0 : find_view_rest(ray_begin, axis_begin, n, s);
    const ViewDev &v = views[vi];
    const int64_t k = s - (ray_begin[vi] - axis_begin[vi]);
    const int64_t left = (int64_t)v.axis_x0 * v.crop_h;
    if (k < left) return pixel_in_columns(v, k, 0, v.axis_x0, tw, th);
    return pixel_in_columns(v, k - left, v.axis_x1, v.crop_w - v.axis_x1, tw, th);
}

// v clamped into FP32's finite range (NaN stays NaN).
__device__ __forceinline__ double sat_double(double v) {
    return isnan(v) ? v : fmax(fmin(v, (double)FLT_MAX), -(double)FLT_MAX);
}
__device__ __forceinline__ float sat_float(double v) { return (float)sat_double(v); }

// v as an unevaluated float pair hi + lo (hi = v rounded, lo = the remainder).
__device__ __forceinline__ void split(double v, float &hi, float &lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

constexpr double kNearHorizon = 0.1;  // FP64 island: steps that start within 0.1 M of r+
// FP64 island next to the spin axis and at extreme momenta.  A ray that
// grazes the axis meets the clamped sin(theta) = 1e-7 (kerr.py:93), where
// p_theta' ~ p_phi^2 cos / sin^3 throws p_theta to ~1e21; the FP64 method
// carries such a ray on (its squares ~1e42 stay finite), FP32's would overflow
// and end the ray as invalid.  Steps that start within 1e-4 rad of a pole or
// with |p_r| or |p_theta| >= 1e15 therefore run in FP64, and so does any step
// whose FP32 result overflows.
constexpr float kPoleIsland = 1.0e-4f;
constexpr float kMomentumIsland = 1.0e15f;
// Tracer32::step's answer for a step that belongs to an FP64 island.
constexpr int kNeedFp64 = -2;

// ------------------------------------------------------------ FP64 helpers
struct Deriv64 {
    double r, th, ph, pr, pth, H;
};

// kerr.py:86-102, :236-303 in FP64: the reference's metric components and
// their quotient-rule derivatives, with each shared denominator inverted once
// -- 1/Sigma, 1/(Sigma Delta), 1/sin^2 -- rather than fifteen divisions per
// call, and sin / cos from one sincos.  Against the division form this moves
// each evaluation by a few ulps and runs the FP64 traces 2.1-2.3x faster:
// images agree to 2e-12 on pixels that a 1e-12 camera perturbation moves by
// less than 1e-9 (7e-10 at 1e-6), and only such perturbation-sensitive pixels
// differ by more.
__device__ __forceinline__ void rhs64(double r, double th_in, double pr, double pth, double pt, double pphi, double a,
                                       Deriv64 &d) {
    const double th = safe_theta(th_in);
    double s, c;
    sincos(th, &s, &c);
    const double a2 = a * a, r2 = r * r;
    const double sig = r2 + a2 * (c * c);
    const double dlt = r2 - 2.0 * r + a2;
    const double A = (r2 + a2) * (r2 + a2) - a2 * dlt * (s * s);
    const double s2 = fmax(s * s, kEpsTheta * kEpsTheta);
    const double ds2 = 2.0 * s * c;
    const double is = 1.0 / sig, isd = 1.0 / (sig * dlt), is2 = 1.0 / s2;
    const double den = sig * dlt, num = -2.0 * a * r, num2 = dlt - a2 * s2, den3 = den * s2;
    const double isd2 = isd * isd, is_2 = is * is, i3 = isd * is2, i3_2 = i3 * i3;
    // g^{mu nu} (kerr.py:86-102)
    const double g03 = num * isd, g33 = num2 * i3;
    d.r = dlt * is * pr;
    d.th = is * pth;
    d.ph = g03 * pt + g33 * pphi;
    // d/dr (kerr.py:236-282, wrt r)
    {
        const double sig_p = 2.0 * r, dlt_p = 2.0 * r - 2.0;
        const double A_p = 4.0 * r * (r2 + a2) - a2 * dlt_p * s2;
        const double den_p = sig_p * dlt + sig * dlt_p;
        const double g00 = -((A_p * den - A * den_p) * isd2);
        const double g03p = (-2.0 * a * den - num * den_p) * isd2;
        const double g11 = (dlt_p * sig - dlt * sig_p) * is_2;
        const double g22 = -sig_p * is_2;
        const double den3_p = sig_p * dlt * s2 + sig * dlt_p * s2;
        const double g33p = (dlt_p * den3 - num2 * den3_p) * i3_2;
        d.pr = -0.5 * (g00 * pt * pt + 2.0 * g03p * pt * pphi + g11 * pr * pr + g22 * pth * pth + g33p * pphi * pphi);
    }
    // d/dtheta
    {
        const double sig_p = -a2 * ds2;
        const double A_p = -a2 * dlt * ds2;
        const double den_p = sig_p * dlt;
        const double g00 = -((A_p * den - A * den_p) * isd2);
        const double g03p = (-num * den_p) * isd2;
        const double g11 = (-dlt * sig_p) * is_2;
        const double g22 = -sig_p * is_2;
        const double den3_p = sig_p * dlt * s2 + sig * dlt * ds2;
        const double g33p = ((-a2 * ds2) * den3 - num2 * den3_p) * i3_2;
        d.pth = -0.5 * (g00 * pt * pt + 2.0 * g03p * pt * pphi + g11 * pr * pr + g22 * pth * pth + g33p * pphi * pphi);
    }
    d.H = 0.5 * ((-A * isd) * pt * pt + 2.0 * g03 * pt * pphi + dlt * is * pr * pr + is * pth * pth + g33 * pphi * pphi);
}

// ------------------------------------------------------------ FP32 tracer
constexpr float kPiH = 3.14159274101257324f;        // pi rounded to float
constexpr float kPiL = -8.74227765734758577e-8f;    // pi - kPiH
constexpr float kHalfPiF = 1.57079637050628662f;
constexpr float kTwoPiH = 6.28318548202514648f;     // 2 pi rounded to float
constexpr float kTwoPiL = -1.74845553146951715e-7f; // 2 pi - kTwoPiH
constexpr float kEpsF = 1.0e-7f;
constexpr float kTmaxH = (float)(kPi - kEpsTheta);  // pi - eps as a float pair (kerr.py:35-36 upper clamp)
constexpr float kTmaxL = (float)((kPi - kEpsTheta) - (double)kTmaxH);

// sin and cos on [eps, pi/2].  Below x = 1/4 (next to a pole, where the
// metric inverse g^phiphi ~ 1/sin^2 needs sin to full relative precision):
// the Taylor series through x^7 and x^8 (truncation below 1.2e-11 relative),
// by Horner in x^2.  Above it the hardware __sincosf (absolute error about
// 2^-21.4, relative below 1.5e-6 there), at a fraction of the series' cost.
__device__ __forceinline__ void sincos_quadrant(float x, float &s, float &c) {
    if (x < 0.25f) {
        const float u = x * x;
        float ps = fmaf(u, -1.9841269841e-4f, 8.3333333333e-3f);  // -1/7!, 1/5!
        ps = fmaf(u, ps, -1.6666666667e-1f);                        // -1/3!
        s = fmaf(x * u, ps, x);
        float pc = fmaf(u, 2.4801587302e-5f, -1.3888888889e-3f);   // 1/8!, -1/6!
        pc = fmaf(u, pc, 4.1666666667e-2f);                         // 1/4!
        pc = fmaf(u, pc, -0.5f);                                    // -1/2!
        c = fmaf(u, pc, 1.0f);
    } else {
        __sincosf(x, &s, &c);
    }
}

// sin(theta), cos(theta) from d, the distance of theta from the pole nearer
// at the step start (south: theta = pi - d).  d keeps full relative precision
// next to either pole because it is formed from the compensated theta, which
// is what the near-pole metric inverse (g^phiphi ~ 1/sin^2) needs.  A
// midpoint may lie past the equator (d > pi/2: x is the distance to the other
// pole) or past the other pole altogether (d > pi - eps, even by many radians
// when p_theta is large): kerr.py:35-36 clips theta into [eps, pi - eps], which
// here is x >= eps, so x never leaves [eps, pi/2] where the series holds.
__device__ __forceinline__ void sincos_pole(float d, bool south, float &s, float &c) {
    const bool over = d > kHalfPiF;  // a half step may cross the equator
    const float x = fmaxf(over ? (kPiH - d) + kPiL : d, kEpsF);
    sincos_quadrant(x, s, c);
    c = (over != south) ? -c : c;
    s = fmaxf(s, kEpsF);  // sin^2 >= eps^2 (kerr.py:93)
}

// hi + lo += d (Kahan's compensated summation: lo carries what hi lost).
__device__ __forceinline__ void kahan_add(float &hi, float &lo, float d) {
    const float y = d + lo;
    const float t = hi + y;
    lo = y - (t - hi);
    hi = t;
}

// hi + lo += d without the |hi| >= |d| precondition (Knuth's TwoSum).
__device__ __forceinline__ void two_sum_add(float &hi, float &lo, float d) {
    const float s = hi + d;
    const float bb = s - hi;
    const float err = (hi - (s - bb)) + (d - bb);
    hi = s;
    lo += err;
}

struct Deriv32 {
    float r, th, ph, pr, pth, H;
};

// Hamiltonian equations of kerr.py:285-303 written through
//   2 Sigma H = F = Delta p_r^2 + p_theta^2 + P^2 - W^2 / Delta,
//   P = p_phi / sin + a sin p_t,  W = (r^2 + a^2) p_t + a p_phi,
// which is g^{mu nu} p_mu p_nu of kerr.py:86-102 regrouped; x' = dH/dp and
// p' = -dH/dx are its exact derivatives (the quotient-rule sums of
// kerr.py:236-282 collapse to these few terms).  With Q = W / Delta and
// G = F / Sigma (= 2H):
//   p_r'     = [(1 - r)(p_r^2 + Q^2) + r (2 p_t Q + G)] / Sigma,
//   p_theta' = cos [P (p_phi / sin^2 - a p_t) - G a^2 sin] / Sigma.
// Delta is formed as (r - r+)(r - r-) from the compensated horizon distance
// x = r - r+, since r^2 - 2r + a^2 cancels to nothing in FP32 next to the
// horizon.
__device__ __forceinline__ void rhs32(float r, float x, float s, float c, float pr, float pth, float pt, float pphi,
                                      float a, float a2, float dpm, Deriv32 &d) {
    const float r2 = r * r;
    const float D = x * (x + dpm);
    const float Sg = fmaf(a2 * c, c, r2);
    const float iS = 1.0f / Sg;
    const float iD = 1.0f / D;
    const float is = 1.0f / s;
    const float W = fmaf(r2 + a2, pt, a * pphi);
    const float P = fmaf(a * pt, s, pphi * is);
    const float Q = W * iD;
    const float Dpr = D * pr;
    const float F = fmaf(Dpr, pr, fmaf(pth, pth, fmaf(P, P, -W * Q)));
    const float G = F * iS;
    d.r = Dpr * iS;
    d.th = pth * iS;
    d.ph = fmaf(P, is, -a * Q) * iS;
    d.pr = fmaf(1.0f - r, fmaf(pr, pr, Q * Q), r * fmaf(pt + pt, Q, G)) * iS;
    d.pth = c * fmaf(P, fmaf(pphi * is, is, -a * pt), -G * (a2 * s)) * iS;
    d.H = 0.5f * G;
}

// rhs32's Hamiltonian form in FP64 (the near-horizon island of the FP32 kernel).
__device__ __forceinline__ void rhs64h(double r, double th_in, double pr, double pth, double pt, double pphi,
                                       double a, double r_plus, double r_minus, Deriv64 &d) {
    const double th = safe_theta(th_in);
    double s, c;
    sincos(th, &s, &c);
    s = fmax(s, kEpsTheta);
    const double a2 = a * a, r2 = r * r;
    const double D = (r - r_plus) * (r - r_minus);
    const double Sg = r2 + a2 * c * c;
    const double iS = 1.0 / Sg, iD = 1.0 / D, is = 1.0 / s;
    const double W = (r2 + a2) * pt + a * pphi;
    const double P = pphi * is + a * s * pt;
    const double Q = W * iD;
    const double F = D * pr * pr + pth * pth + P * P - W * Q;
    d.r = D * pr * iS;
    d.th = pth * iS;
    d.ph = (P * is - a * Q) * iS;
    const double dFr = (2.0 * r - 2.0) * (pr * pr + Q * Q) - 4.0 * r * pt * Q;
    d.pr = (-0.5 * dFr + F * r * iS) * iS;
    const double dFth = 2.0 * P * c * (a * pt - pphi * is * is);
    d.pth = (-0.5 * dFth - F * a2 * s * c * iS) * iS;
    d.H = 0.5 * F * iS;
}

// The FP32 tracer's Stokes vector, one slot per thread of the block (render
// blocks have at most 256 threads).  It is read and written only on in-brick
// steps and at the end of the ray, so it need not hold four registers across
// the geodesic loop (which runs at an 80-register budget): 4 % faster.
__shared__ float4 g_stokes[256];

struct Tracer32 {
    static constexpr bool kIslands = true;  // step may answer kNeedFp64
    float rh, rl, th_h, th_l, ph_h, ph_l;  // positions as compensated pairs (value = hi + lo)
    float pr, pth, pt, pphi;
    float tau, drift, H0;
    int steps, brick, vi;
    uint32_t out_idx;

    __device__ __forceinline__ void init(const ViewDev &v, int view, int px, int py, int64_t out_index) {
        const CameraRay c = camera_ray(v, px, py);
        split(v.r_obs, rh, rl);
        split(v.theta_obs, th_h, th_l);
        double p0 = fmod(v.phi_obs, kTwoPi);
        if (p0 < 0.0) p0 += kTwoPi;
        split(p0, ph_h, ph_l);
        pr = (float)c.pr;
        pth = (float)c.pth;
        pt = (float)c.pt;
        pphi = (float)c.pphi;
        H0 = (float)c.H0;
        g_stokes[threadIdx.x] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        tau = 0.0f;
        drift = 0.0f;
        steps = 0;
        brick = 0;
        vi = view;
        out_idx = (uint32_t)out_index;
    }

    // The FP64 island next to the horizon: the whole RK2 step in FP64, since
    // p_r ~ 1/Delta leaves FP32's exponent range there.
    // Returns 0 (finite), 1 (non-finite) or 2 (horizon guard: the midpoint lies
    // inside the horizon; the state is left unchanged).
    // Not inlined: the FP64 step runs for a few steps in a thousand, and keeping
    // its code out of the FP32 loop keeps that loop's registers for itself.  It
    // is only ever called on a copy of the tracer (step64), so the tracer that
    // the FP32 loop carries is never address-taken and stays in registers.
    __device__ __noinline__ int step_fp64(const ViewDev &v, bool guard, float &dr, float &dph) {
        const double r = (double)rh + (double)rl;
        const double th = (double)th_h + (double)th_l;
        const double ph = (double)ph_h + (double)ph_l;
        const double h = fmin(fmax(v.h_scale * r, v.h_min), v.h_max);
        Deriv64 k1, k2;
        rhs64h(r, th, pr, pth, pt, pphi, v.a, v.r_plus, v.r_minus, k1);
        drift = fmaxf(drift, (float)fabs(fabs(k1.H) - (double)H0));
        const double hh = 0.5 * h;
        if (guard && r + hh * k1.r < v.r_plus) return 2;
        rhs64h(r + hh * k1.r, th + hh * k1.th, pr + hh * k1.pr, pth + hh * k1.pth, pt, pphi, v.a, v.r_plus,
               v.r_minus, k2);
        const double rn = r + h * k2.r, thn = safe_theta(th + h * k2.th), phn = ph + h * k2.ph;
        const double prn = pr + h * k2.pr, pthn = pth + h * k2.pth;
        // a catastrophic step of the reference's method (a ray flung off the pole
        // or out of the horizon) can leave FP32's range while FP64 stays finite:
        // such values are kept saturated at +-FLT_MAX, which ends the ray with
        // the FP64 method's status (captured at r -> -inf, escaped at r -> +inf)
        dr = sat_float(rn - r);
        dph = sat_float(phn - ph);
        split(sat_double(rn), rh, rl);
        split(thn, th_h, th_l);
        split(sat_double(phn), ph_h, ph_l);
        pr = sat_float(prn);
        pth = sat_float(pthn);
        return (isfinite(rn) && isfinite(thn) && isfinite(phn) && isfinite(prn) && isfinite(pthn)) ? 0 : 1;
    }

    // One RK2 geodesic step plus its brick segment.  Returns -1 while the ray
    // lives, kNeedFp64 (state untouched) when the step belongs to an FP64
    // island -- the caller then takes it with step64, outside its FP32 loop --
    // else the ray's BHN_RAY_* status.
    __device__ __forceinline__ int step(const StepConst &C, const Tables &T, const float4 *__restrict__ rec, int nr,
                                        int nt, int np, const ViewDev *__restrict__ views) {
        if (rh < C.r_guard && pr < 0.0f) return BHN_RAY_CAPTURED;  // horizon guard (flag; off by default)
        const float r0 = rh + rl, th0 = th_h + th_l, ph0 = ph_h + ph_l;
        float dr = 0.0f, dph = 0.0f;
        const bool south = th_h > kHalfPiF;
        const float d0 = south ? (kPiH - th_h) + (kPiL - th_l) : th0;
        bool fp64 = rh < C.r_near || d0 < kPoleIsland || !(fabsf(pth) < kMomentumIsland && fabsf(pr) < kMomentumIsland);
        if (!fp64) {
            float s, c;
            sincos_pole(d0, south, s, c);
            const float x0 = (rh - C.rp_h) + (rl - C.rp_l);
            const float h = fminf(fmaxf(C.hs * r0, C.hmin), C.hmax);
            Deriv32 k1;
            rhs32(r0, x0, s, c, pr, pth, pt, pphi, C.a, C.a2, C.dpm, k1);
            drift = fmaxf(drift, fabsf(fabsf(k1.H) - H0));
            const float hh = 0.5f * h;
            // horizon guard: a step whose midpoint lies inside the horizon is not taken
            if (C.r_guard > 0.0f && fmaf(hh, k1.r, x0) < 0.0f) return BHN_RAY_CAPTURED;
            // midpoint: pole distance clamped at eps like kerr.py:35-36 inside the right-hand side
            const float dm = fmaxf(south ? fmaf(-hh, k1.th, d0) : fmaf(hh, k1.th, d0), kEpsF);
            sincos_pole(dm, south, s, c);
            Deriv32 k2;
            rhs32(fmaf(hh, k1.r, r0), fmaf(hh, k1.r, x0), s, c, fmaf(hh, k1.pr, pr), fmaf(hh, k1.pth, pth), pt, pphi,
                  C.a, C.a2, C.dpm, k2);
            dr = h * k2.r;
            const float dth = h * k2.th;
            dph = h * k2.ph;
            const float prn = fmaf(h, k2.pr, pr), pthn = fmaf(h, k2.pth, pth);
            // An FP32 overflow here (a ray flung off the pole or out of the
            // horizon reaches momenta of 1e30 and more, whose squares FP64 still
            // holds) sends the step to FP64, from the untouched start state.
            fp64 = !isfinite(dr + dth + dph + prn + pthn);
            if (!fp64) {
                kahan_add(rh, rl, dr);
                kahan_add(th_h, th_l, dth);
                kahan_add(ph_h, ph_l, dph);
                pr = prn;
                pth = pthn;
                // theta clamp (kerr.py:312)
                if (th_h + th_l < kEpsF) {
                    th_h = kEpsF;
                    th_l = 0.0f;
                } else if ((th_h - kTmaxH) + (th_l - kTmaxL) > 0.0f) {
                    th_h = kTmaxH;
                    th_l = kTmaxL;
                }
            }
        }
        if (fp64) return kNeedFp64;
        return segment(C, T, rec, nr, nt, np, r0, th0, ph0, dr, dph, true);
    }

    // The step in FP64 (an island), then its brick segment; returns like step.
    __device__ __forceinline__ int step64(const StepConst &C, const Tables &T, const float4 *__restrict__ rec, int nr,
                                          int nt, int np, const ViewDev *__restrict__ views) {
        const float r0 = rh + rl, th0 = th_h + th_l, ph0 = ph_h + ph_l;
        float dr = 0.0f, dph = 0.0f;
        Tracer32 t = *this;
        const int rc = t.step_fp64(views[vi], C.r_guard > 0.0f, dr, dph);
        *this = t;
        if (rc == 2) return BHN_RAY_CAPTURED;
        return segment(C, T, rec, nr, nt, np, r0, th0, ph0, dr, dph, rc == 0);
    }

    // Everything after the geodesic update: the step count, phi back into
    // [0, 2 pi), the segment from (r0, th0, ph0) to the new state, and the
    // stopping rules.
    __device__ __forceinline__ int segment(const StepConst &C, const Tables &T, const float4 *__restrict__ rec, int nr,
                                           int nt, int np, float r0, float th0, float ph0, float dr, float dph,
                                           bool finite) {
        ++steps;
        const float th1 = th_h + th_l;
        // phi is only sampled modulo 2 pi: keep the state in [0, 2 pi)
        if (ph_h >= kTwoPiH) {
            two_sum_add(ph_h, ph_l, -kTwoPiH);
            ph_l -= kTwoPiL;
        } else if (ph_h < 0.0f) {
            two_sum_add(ph_h, ph_l, kTwoPiH);
            ph_l += kTwoPiL;
        }

        // segment (y, y_n): accelerated_renderer.py:113-125
        if (tau < C.max_tau) {
            const float rmid = fmaf(0.5f, dr, r0), tmid = 0.5f * (th0 + th1), pmid = fmaf(0.5f, dph, ph0);
            // nonperiodic valid mask (native_kernels.py:189-210); NaN passes it as in the reference
            if (!(rmid < T.grf[0] || rmid > T.grf[nr - 1]) && !(tmid < T.gtf[0] || tmid > T.gtf[nt - 1])) {
                ++brick;
                if (!(isfinite(rmid) && isfinite(tmid) && isfinite(pmid))) {
                    // NaN coefficients in the reference -> NaN Stokes -> nan_to_num -> 0
                    const float qnan = __int_as_float(0x7fc00000);
                    g_stokes[threadIdx.x] = make_float4(qnan, qnan, qnan, qnan);
                } else {
                    const TableHeader &H = *T.h;
                    const float g0 = T.gpf[0];
                    float pw = pmid - g0;
                    pw = fmaf(-kTwoPiH, floorf(pw * 0.159154943f), pw) + g0;  // wrap into [g0, g0 + 2 pi)
                    pw = fmaxf(pw, g0);
                    const int ir = locate_linear_f(T.grf, nr, rmid, H.kind_r, H.foff_r, H.finv_r);
                    const int it = locate_linear_f(T.gtf, nt, tmid, H.kind_t, H.foff_t, H.finv_t);
                    const int ip = locate_phi_f(T.gpf, np, pw, H.kind_p, H.foff_p, H.finv_p);
                    const int ip1 = ip + 1 == np ? 0 : ip + 1;
                    const float wr = (rmid - T.grf[ir]) * T.idr[ir];
                    const float wt = (tmid - T.gtf[it]) * T.idt[it];
                    const float wp = (pw - T.gpf[ip]) * T.idp[ip];
                    const float owr = 1.0f - wr, owt = 1.0f - wt, owp = 1.0f - wp;
                    // 32-bit cell offsets (launch_render admits bricks of < 2^32 float4 records)
                    const uint32_t c00 = ((uint32_t)ir * nt + it) * np;
                    const uint32_t cells[4] = {c00, c00 + np, c00 + (uint32_t)(nt * np), c00 + (uint32_t)(nt * np + np)};
                    const float wrt[4] = {owr * owt, owr * wt, wr * owt, wr * wt};
                    // channels in pairs on the paired FP32 FMA (each lane one fmaf, same order)
                    float2 c01 = make_float2(0.0f, 0.0f), c23 = c01, c45 = c01, c67 = c01, c89 = c01;
                    float c10 = 0.0f;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 *p0 = rec + 3u * (cells[q] + (uint32_t)ip);
                        const float4 *p1 = rec + 3u * (cells[q] + (uint32_t)ip1);
                        const float w0 = wrt[q] * owp, w1 = wrt[q] * wp;
                        const float2 W0 = make_float2(w0, w0), W1 = make_float2(w1, w1);
                        const float4 a0 = __ldg(p0), b0 = __ldg(p0 + 1), c0 = __ldg(p0 + 2);
                        const float4 a1 = __ldg(p1), b1 = __ldg(p1 + 1), c1 = __ldg(p1 + 2);
                        c01 = __ffma2_rn(W0, make_float2(a0.x, a0.y), __ffma2_rn(W1, make_float2(a1.x, a1.y), c01));
                        c23 = __ffma2_rn(W0, make_float2(a0.z, a0.w), __ffma2_rn(W1, make_float2(a1.z, a1.w), c23));
                        c45 = __ffma2_rn(W0, make_float2(b0.x, b0.y), __ffma2_rn(W1, make_float2(b1.x, b1.y), c45));
                        c67 = __ffma2_rn(W0, make_float2(b0.z, b0.w), __ffma2_rn(W1, make_float2(b1.z, b1.w), c67));
                        c89 = __ffma2_rn(W0, make_float2(c0.x, c0.y), __ffma2_rn(W1, make_float2(c1.x, c1.y), c89));
                        c10 = fmaf(w0, c0.z, fmaf(w1, c1.z, c10));
                    }
                    const float cf[11] = {c01.x, c01.y, c23.x, c23.y, c45.x, c45.y, c67.x, c67.y, c89.x, c89.y, c10};
                    // ds = L * max(|d(r, theta, phi)|, 1e-14) (accelerated_renderer.py:120-121)
                    const float dth = th1 - th0;
                    const float ds = C.L * fmaxf(sqrtf(fmaf(dr, dr, fmaf(dth, dth, dph * dph))), 1.0e-14f);
                    // Stokes RK2 (lib.rs:210-225) with K of native_kernels.py:213-222
                    const float j0 = cf[0], j1 = cf[1], j2 = cf[2], j3 = cf[3];
                    const float ai = cf[4], aq = cf[5], au = cf[6], av = cf[7];
                    const float rv = cf[8], rq = cf[9], ru = cf[10];
                    float S0, S1, S2, S3;
                    {
                        const float4 Sv = g_stokes[threadIdx.x];
                        S0 = Sv.x, S1 = Sv.y, S2 = Sv.z, S3 = Sv.w;
                    }
                    float k0 = j0 - (ai * S0 + aq * S1 + au * S2 + av * S3);
                    float kq = j1 - (aq * S0 + ai * S1 + rv * S2 - ru * S3);
                    float ku = j2 - (au * S0 - rv * S1 + ai * S2 + rq * S3);
                    float kv = j3 - (av * S0 + ru * S1 - rq * S2 + ai * S3);
                    const float hd = 0.5f * ds;
                    const float m0 = fmaf(hd, k0, S0), m1 = fmaf(hd, kq, S1), m2 = fmaf(hd, ku, S2),
                                m3 = fmaf(hd, kv, S3);
                    k0 = j0 - (ai * m0 + aq * m1 + au * m2 + av * m3);
                    kq = j1 - (aq * m0 + ai * m1 + rv * m2 - ru * m3);
                    ku = j2 - (au * m0 - rv * m1 + ai * m2 + rq * m3);
                    kv = j3 - (av * m0 + ru * m1 - rq * m2 + ai * m3);
                    S0 = fmaf(ds, k0, S0);
                    S1 = fmaf(ds, kq, S1);
                    S2 = fmaf(ds, ku, S2);
                    S3 = fmaf(ds, kv, S3);
                    g_stokes[threadIdx.x] = make_float4(S0, S1, S2, S3);
                    tau = fmaf(fmaxf(ai, 0.0f), ds, tau);
                }
            }
        }
        // kerr.py:364-377
        if (!finite) return BHN_RAY_INVALID;
        if (tau >= C.max_tau) return BHN_RAY_OPAQUE;
        if ((rh - C.rcap_h) + (rl - C.rcap_l) <= 0.0f) return BHN_RAY_CAPTURED;
        if (rh > C.esc && dr > 0.0f) return BHN_RAY_ESCAPED;
        if (steps >= C.max_steps) return BHN_RAY_MAX_STEPS;
        return -1;
    }

    __device__ __forceinline__ void finish(void *out, int status, const StepConst &C, const ViewDev *views) {
        if (status != BHN_RAY_INVALID) {  // drift at the final state (kerr.py:360, 367)
            const bool south = th_h > kHalfPiF;
            const float d0 = south ? (kPiH - th_h) + (kPiL - th_l) : th_h + th_l;
            if (rh < C.r_near || d0 < kPoleIsland ||
                !(fabsf(pth) < kMomentumIsland && fabsf(pr) < kMomentumIsland && fabsf(rh) < kMomentumIsland)) {
                // a state the FP32 right-hand side cannot evaluate (the islands, or a
                // ray flung to |r| >= 1e15 by its last step): H in FP64
                const ViewDev &v = views[vi];
                Deriv64 k;
                rhs64h((double)rh + (double)rl, (double)th_h + (double)th_l, pr, pth, pt, pphi, v.a, v.r_plus,
                       v.r_minus, k);
                drift = fmaxf(drift, (float)fmin(fabs(fabs(k.H) - (double)H0), (double)FLT_MAX));
            } else {
                float s, c;
                sincos_pole(d0, south, s, c);
                Deriv32 k;
                rhs32(rh + rl, (rh - C.rp_h) + (rl - C.rp_l), s, c, pr, pth, pt, pphi, C.a, C.a2, C.dpm, k);
                drift = fmaxf(drift, fabsf(fabsf(k.H) - H0));
            }
        }
        // np.nan_to_num(S, nan=0, posinf=0, neginf=0) (accelerated_renderer.py:126)
        float4 o;
        const float4 S = g_stokes[threadIdx.x];
        o.x = isfinite(S.x) ? S.x : 0.0f;
        o.y = isfinite(S.y) ? S.y : 0.0f;
        o.z = isfinite(S.z) ? S.z : 0.0f;
        o.w = isfinite(S.w) ? S.w : 0.0f;
        reinterpret_cast<float4 *>(out)[out_idx] = o;
    }

    // The drift output is a float: drifts beyond its range (a catastrophic last
    // step can reach 1e60 in FP64) are stored as FLT_MAX.
    __device__ __forceinline__ float drift_f() const { return fminf(drift, FLT_MAX); }

    static __device__ __forceinline__ void write_zero(void *out, int64_t idx) {
        reinterpret_cast<float4 *>(out)[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
};

// ------------------------------------------------------------ FP64 tracer
struct Tracer64 {
    static constexpr bool kIslands = false;  // step never answers kNeedFp64
    double r, th, ph, pr, pth, pt, pphi;
    double S0, S1, S2, S3, tau, drift, H0;
    int steps, brick, vi;
    bool poison;
    uint32_t out_idx;

    __device__ __forceinline__ void init(const ViewDev &v, int view, int px, int py, int64_t out_index) {
        const CameraRay c = camera_ray(v, px, py);
        r = v.r_obs;
        th = v.theta_obs;
        ph = v.phi_obs;
        pr = c.pr;
        pth = c.pth;
        pt = c.pt;
        pphi = c.pphi;
        H0 = c.H0;
        S0 = S1 = S2 = S3 = 0.0;
        tau = 0.0;
        drift = 0.0;
        steps = 0;
        brick = 0;
        vi = view;
        poison = false;
        out_idx = (uint32_t)out_index;
    }

    __device__ __forceinline__ int step(const StepConst &C, const Tables &T, const double2 *__restrict__ rec, int nr,
                                        int nt, int np, const ViewDev *__restrict__ views) {
        const ViewDev &v = views[vi];
        if (C.r_guard > 0.0f && r < fmin(v.r_photon, T.gr[0]) && pr < 0.0) return BHN_RAY_CAPTURED;
        const double h = fmin(fmax(v.h_scale * r, v.h_min), v.h_max);
        Deriv64 k1, k2;
        rhs64(r, th, pr, pth, pt, pphi, v.a, k1);
        drift = fmax(drift, fabs(fabs(k1.H) - H0));
        const double hh = 0.5 * h;
        // horizon guard: a step whose midpoint lies inside the horizon is not taken
        if (C.r_guard > 0.0f && r + hh * k1.r < v.r_plus) return BHN_RAY_CAPTURED;
        rhs64(r + hh * k1.r, th + hh * k1.th, pr + hh * k1.pr, pth + hh * k1.pth, pt, pphi, v.a, k2);
        const double rn = r + h * k2.r;
        const double thn = safe_theta(th + h * k2.th);
        const double phn = ph + h * k2.ph;
        pr = pr + h * k2.pr;
        pth = pth + h * k2.pth;
        ++steps;
        const bool finite = isfinite(rn) && isfinite(thn) && isfinite(phn) && isfinite(pr) && isfinite(pth);
        if (tau < v.max_tau) {
            const double rmid = 0.5 * (r + rn), tmid = 0.5 * (th + thn), pmid = 0.5 * (ph + phn);
            const TableHeader &H = *T.h;
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
                    double ds = v.L * dl;
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
        if (tau >= v.max_tau) return BHN_RAY_OPAQUE;
        if (rn <= v.r_capture) return BHN_RAY_CAPTURED;
        if (rn > v.escape_radius && rn > r_old) return BHN_RAY_ESCAPED;
        if (steps >= v.max_steps) return BHN_RAY_MAX_STEPS;
        return -1;
    }

    __device__ __forceinline__ void finish(void *out, int status, const StepConst &C, const ViewDev *views) {
        if (status != BHN_RAY_INVALID) {
            Deriv64 k;
            rhs64(r, th, pr, pth, pt, pphi, views[vi].a, k);
            drift = fmax(drift, fabs(fabs(k.H) - H0));
        }
        double2 *o = reinterpret_cast<double2 *>(out) + 2 * (int64_t)out_idx;
        o[0] = make_double2((poison || !isfinite(S0)) ? 0.0 : S0, (poison || !isfinite(S1)) ? 0.0 : S1);
        o[1] = make_double2((poison || !isfinite(S2)) ? 0.0 : S2, (poison || !isfinite(S3)) ? 0.0 : S3);
    }

    __device__ __forceinline__ float drift_f() const { return (float)fmin(drift, (double)FLT_MAX); }

    static __device__ __forceinline__ void write_zero(void *out, int64_t idx) {
        double2 *o = reinterpret_cast<double2 *>(out) + 2 * idx;
        o[0] = make_double2(0.0, 0.0);
        o[1] = make_double2(0.0, 0.0);
    }
};

template <class T> struct RecordOf;
template <> struct RecordOf<Tracer32> { using type = float4; };
template <> struct RecordOf<Tracer64> { using type = double2; };

__host__ __device__ inline int64_t align16(int64_t x) { return (x + 15) & ~(int64_t)15; }

// Shared-memory layout of the persistent kernel.
__host__ __device__ inline int64_t smem_bytes(int tables_bytes, int n_views) {
    return align16(tables_bytes) + align16(8 * ((int64_t)n_views + 1)) + (int64_t)sizeof(StepConst) * n_views +
           align16(sizeof(BlockCounters)) + align16(8 * ((int64_t)n_views + 1));
}

// ------------------------------------------------------------ persistent loop
// MINB = resident 256-thread blocks the register allocation must allow:
// 1 -> unconstrained, 3 -> <= 85 registers, 4 -> <= 64 registers.
template <class Tracer, int MINB, bool BATCH>
__global__ void __launch_bounds__(256, MINB) render_kernel(const RenderParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    int64_t *vbegin = reinterpret_cast<int64_t *>(smem + align16(P.tables_bytes));
    StepConst *sconst = reinterpret_cast<StepConst *>(smem + align16(P.tables_bytes) + align16(8 * (P.n_views + 1)));
    BlockCounters *bc = reinterpret_cast<BlockCounters *>(sconst + P.n_views);
    int64_t *abegin = reinterpret_cast<int64_t *>(reinterpret_cast<unsigned char *>(bc) + align16(sizeof(BlockCounters)));
    // grid tables, the view prefix and the per-view step constants stay in shared memory for the launch
    {
        const int4 *src = reinterpret_cast<const int4 *>(P.tables);
        int4 *dst = reinterpret_cast<int4 *>(smem);
        for (int i = threadIdx.x; i < P.tables_bytes / 16; i += blockDim.x) dst[i] = src[i];
        for (int i = threadIdx.x; i <= P.n_views; i += blockDim.x) {
            vbegin[i] = P.ray_begin[i];
            abegin[i] = P.axis_begin[i];
        }
        if (threadIdx.x == 0) memset(bc, 0, sizeof(BlockCounters));
    }
    __syncthreads();
    const Tables T = tables_at(smem, P.nr, P.nt, P.np);
    for (int i = threadIdx.x; i < P.n_views; i += blockDim.x) {
        const ViewDev &v = P.views[i];
        StepConst c;
        c.a = (float)v.a;
        c.a2 = c.a * c.a;
        c.dpm = (float)(v.r_plus - v.r_minus);
        c.hs = (float)v.h_scale;
        c.hmin = (float)v.h_min;
        c.hmax = (float)v.h_max;
        c.L = (float)v.L;
        c.max_tau = (float)v.max_tau;
        split(v.r_plus, c.rp_h, c.rp_l);
        split(v.r_capture, c.rcap_h, c.rcap_l);
        c.esc = (float)v.escape_radius;
        c.r_guard = (v.flags & BHN_VIEW_HORIZON_GUARD) ? (float)fmin(v.r_photon, T.gr[0]) : 0.0f;
        c.r_near = (float)(v.r_plus + kNearHorizon);
        c.pad = 0.0f;
        c.max_steps = v.max_steps;
        c.pad1 = c.pad2 = c.pad3 = 0;
        sconst[i] = c;
    }
    __syncthreads();
    const unsigned long long total = vbegin[P.n_views];
    using Rec = typename RecordOf<Tracer>::type;
    const Rec *rec = reinterpret_cast<const Rec *>(P.records);

    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    Tracer tr;
    bool alive = false, exhausted = BATCH;

    // Batch mode (refill_min = 32): a warp takes 32 consecutive ray slots with one
    // atomic and every lane traces its ray to the end in a tight loop; the warp
    // fetches again once all 32 are done.  No per-step warp vote.
    while (BATCH) {
        unsigned long long base = 0;
        if (lane == 0) {
            base = atomicAdd(&P.q->next, 32ull);
            atomicAdd(&bc->fetches, 1ull);
        }
        base = __shfl_sync(kFull, base, 0);
        if (base >= total) break;
        const unsigned long long slot = base + lane;
        if (slot < total) {
            int vi;
            const PixelRef px = ordered_pixel(P.views, vbegin, abegin, P.n_views, (int64_t)slot, P.tile_w, P.tile_h, vi);
            const ViewDev &v = P.views[vi];
            if (v.valid && v.max_steps > 0) {
                tr.init(v, vi, px.px, px.py, px.out_idx);
                const StepConst &C = sconst[vi];
                int st;
                // the FP32 steps in a tight inner loop; an island step leaves it
                // for the out-of-line FP64 step and comes back
                for (;;) {
                    do {
                        st = tr.step(C, T, rec, P.nr, P.nt, P.np, P.views);
                    } while (st == -1);
                    if constexpr (Tracer::kIslands) {
                        if (st != kNeedFp64) break;
                        st = tr.step64(C, T, rec, P.nr, P.nt, P.np, P.views);
                        if (st != -1) break;
                    } else {
                        break;
                    }
                }
                tr.finish(P.out, st, C, P.views);
                const float d = tr.drift_f();
                atomicAdd(&bc->steps, (unsigned long long)tr.steps);
                atomicAdd(&bc->brick, (unsigned long long)tr.brick);
                atomicAdd(&bc->rays, 1u);
                atomicAdd(&bc->status[st], 1u);
                atomicMax(reinterpret_cast<unsigned int *>(&bc->max_drift), __float_as_uint(d));
                if (st == BHN_RAY_ESCAPED)
                    atomicMax(reinterpret_cast<unsigned int *>(&bc->max_drift_escaped), __float_as_uint(d));
                if (P.ray_steps) P.ray_steps[tr.out_idx] = tr.steps;
                if (P.ray_status) P.ray_status[tr.out_idx] = (uint8_t)st;
                if (P.ray_drift) P.ray_drift[tr.out_idx] = d;
            } else {
                Tracer::write_zero(P.out, px.out_idx);
                const int zst = v.valid ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID;
                atomicAdd(&bc->rays, 1u);
                atomicAdd(&bc->status[zst], 1u);
                if (P.ray_steps) P.ray_steps[px.out_idx] = 0;
                if (P.ray_status) P.ray_status[px.out_idx] = (uint8_t)zst;
                if (P.ray_drift) P.ray_drift[px.out_idx] = 0.0f;
            }
        }
        __syncwarp();
    }

    // Compaction mode (refill_min < 32): every step, the warp votes; once
    // refill_min lanes are done it refills them with one atomic (ballot + popc).
    while (!BATCH && (!exhausted || __any_sync(kFull, alive))) {
        const unsigned dead = __ballot_sync(kFull, !alive);
        const int ndead = __popc(dead);
        if (!exhausted && ndead > 0 && (ndead >= P.refill_min || ndead == 32)) {
            unsigned long long base = 0;
            if (lane == 0) {
                base = atomicAdd(&P.q->next, (unsigned long long)ndead);
                atomicAdd(&bc->fetches, 1ull);
            }
            base = __shfl_sync(kFull, base, 0);
            if (base + (unsigned long long)ndead >= total) exhausted = true;
            if (!alive) {
                const unsigned long long slot = base + __popc(dead & lt_mask);
                if (slot < total) {
                    int vi;
                    const PixelRef px =
                        ordered_pixel(P.views, vbegin, abegin, P.n_views, (int64_t)slot, P.tile_w, P.tile_h, vi);
                    const ViewDev &v = P.views[vi];
                    if (v.valid && v.max_steps > 0) {
                        tr.init(v, vi, px.px, px.py, px.out_idx);
                        alive = true;
                    } else {
                        // no step is taken: the reference returns a zero Stokes vector
                        Tracer::write_zero(P.out, px.out_idx);
                        const int zst = v.valid ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID;
                        atomicAdd(&bc->rays, 1u);
                        atomicAdd(&bc->status[zst], 1u);
                        if (P.ray_steps) P.ray_steps[px.out_idx] = 0;
                        if (P.ray_status) P.ray_status[px.out_idx] = (uint8_t)zst;
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
            const StepConst &C = sconst[tr.vi];
            int st = tr.step(C, T, rec, P.nr, P.nt, P.np, P.views);
            if constexpr (Tracer::kIslands) {
                if (st == kNeedFp64) st = tr.step64(C, T, rec, P.nr, P.nt, P.np, P.views);
            }
            if (st >= 0) {
                tr.finish(P.out, st, C, P.views);
                const float d = tr.drift_f();
                atomicAdd(&bc->steps, (unsigned long long)tr.steps);
                atomicAdd(&bc->brick, (unsigned long long)tr.brick);
                atomicAdd(&bc->rays, 1u);
                atomicAdd(&bc->status[st], 1u);
                atomicMax(reinterpret_cast<unsigned int *>(&bc->max_drift), __float_as_uint(d));
                if (st == BHN_RAY_ESCAPED)
                    atomicMax(reinterpret_cast<unsigned int *>(&bc->max_drift_escaped), __float_as_uint(d));
                if (P.ray_steps) P.ray_steps[tr.out_idx] = tr.steps;
                if (P.ray_status) P.ray_status[tr.out_idx] = (uint8_t)st;
                if (P.ray_drift) P.ray_drift[tr.out_idx] = d;
                alive = false;
            }
        }
    }

    // block totals -> launch totals (non-negative floats order like their bit patterns)
    __syncthreads();
    if (threadIdx.x == 0 && P.stats) {
        atomicAdd(&P.stats->ray_steps, bc->steps);
        atomicAdd(&P.stats->brick_steps, bc->brick);
        atomicAdd(&P.stats->rays, (unsigned long long)bc->rays);
        for (int k = 0; k < 5; ++k)
            if (bc->status[k]) atomicAdd(&P.stats->status[k], (unsigned long long)bc->status[k]);
        atomicAdd(&P.stats->queue_fetches, bc->fetches);
        atomicMax(reinterpret_cast<unsigned int *>(&P.stats->max_h_drift), __float_as_uint(bc->max_drift));
        atomicMax(reinterpret_cast<unsigned int *>(&P.stats->max_h_drift_escaped),
                  __float_as_uint(bc->max_drift_escaped));
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
    if (cfg->reg_cap != 0 && cfg->reg_cap != 80 && cfg->reg_cap != 64)
        return fail(BHN_ERR_VALUE, "reg_cap must be 0, 80 or 64");
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
    if (cfg->precision == 0 && 3 * (int64_t)nr * nt * np >= ((int64_t)1 << 32))
        return fail(BHN_ERR_VALUE, "the FP32 kernel takes bricks of fewer than 2^32 / 3 cells (32-bit record offsets)");
    ScratchLayout L = scratch_layout(n_views);
    if (scratch_bytes < L.total) return fail(BHN_ERR_VALUE, "scratch buffer is smaller than bhn_render_scratch_bytes()");
    if (reinterpret_cast<uintptr_t>(records) % 16 || reinterpret_cast<uintptr_t>(tables) % 16 ||
        reinterpret_cast<uintptr_t>(scratch) % 256 || reinterpret_cast<uintptr_t>(out) % 16)
        return fail(BHN_ERR_VALUE, "records/tables/out must be 16-byte and scratch 256-byte aligned");
    const int tables_bytes = (int)table_layout(nr, nt, np).total;
    const int64_t smem64 = smem_bytes(tables_bytes, n_views);
    if (smem64 > 200 * 1024) return fail(BHN_ERR_VALUE, "brick grids plus views exceed the shared-memory table budget");
    const int smem = (int)smem64;
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
    P.axis_begin = reinterpret_cast<const int64_t *>(sc + L.axis_begin);
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
    auto go = [&](auto kernel) -> int {
        if (smem > 48 * 1024)
            BHN_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kernel<<<grid, block, smem, s>>>(P);
        BHN_LAUNCH_CHECK("render_kernel");
        return BHN_OK;
    };
    const bool batch = cfg->refill_min >= 32;
    if (cfg->precision == 1) return batch ? go(render_kernel<Tracer64, 1, true>) : go(render_kernel<Tracer64, 1, false>);
    if (cfg->reg_cap == 64) return batch ? go(render_kernel<Tracer32, 4, true>) : go(render_kernel<Tracer32, 4, false>);
    if (cfg->reg_cap == 80) return batch ? go(render_kernel<Tracer32, 3, true>) : go(render_kernel<Tracer32, 3, false>);
    return batch ? go(render_kernel<Tracer32, 1, true>) : go(render_kernel<Tracer32, 1, false>);
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
        // the kernels keep a ray's output index in 32 bits
        if (v.out_offset + (int64_t)v.crop_w * v.crop_h > ((int64_t)1 << 32))
            return fail(BHN_ERR_VALUE, "views address more than 2^32 output pixels");
    }
    cudaStream_t s = as_stream(stream);
    char *sc = static_cast<char *>(scratch);
    BHN_CUDA_TRY(cudaMemcpyAsync(sc + L.raw_views, h_views, sizeof(bhn_view) * n_views, cudaMemcpyHostToDevice, s));
    setup_views_kernel<<<1, 256, 0, s>>>(reinterpret_cast<const bhn_view *>(sc + L.raw_views), n_views,
                                         reinterpret_cast<ViewDev *>(sc + L.views),
                                         reinterpret_cast<int64_t *>(sc + L.ray_begin),
                                         reinterpret_cast<int64_t *>(sc + L.axis_begin),
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
#include "bhn_learned.cuh"
#include "bhn_grrt.cuh"
#include "bhn_bricktrace.cuh"
