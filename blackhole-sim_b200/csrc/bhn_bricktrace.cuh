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
// Python's method: one thread per ray (brick_trace_kernel), or, for images of
// at most 4 ray warps per SM, two warps per 32 rays (brick_trace_pair_kernel:
// a geodesic warp and a transfer warp joined by an mbarrier ring).  A ray
// past the brick's outer radius moving out for good also ends
// (outbound_for_good, bhn_grrt.cuh): nothing later is sampled.

#include "bhn_exact.cuh"
#include "bhn_transfer.cuh"

namespace bhn {

struct BrickTraceParams {
    const void *coeffs;          // [nr][nt][np][11] float64, or 12-wide cell records (BHN_BRICK_*)
    const double *rg, *tg, *pg;
    int nr, nt, np, max_steps, exact_step, full_trace;
    const ViewDev *view;
    double step, escape_radius, length_cm, max_tau;
    double *out;                 // [rays][4]
    double *diag;                // optional [rays][4]: optical depth, sampled segments, steps, status
};

// One cell sample in the brick's layout: the 11-channel float64 brick as the
// reference holds it, or its 12-wide float32 / float64 cell records.
template <int Layout>
__device__ __forceinline__ bool sample_brick(const BrickTraceParams &P, const AxisHints &h, double r, double th,
                                             double ph, double c[11]) {
    if constexpr (Layout == BHN_BRICK_F32X12)
        return sample_weighted_hinted<float, 12>(static_cast<const float *>(P.coeffs), P.rg, P.nr, P.tg, P.nt, P.pg,
                                                 P.np, h, r, th, ph, c);
    else if constexpr (Layout == BHN_BRICK_F64X12)
        return sample_weighted_hinted<double, 12>(static_cast<const double *>(P.coeffs), P.rg, P.nr, P.tg, P.nt, P.pg,
                                                  P.np, h, r, th, ph, c);
    else
        return sample_weighted_hinted<double, 11>(static_cast<const double *>(P.coeffs), P.rg, P.nr, P.tg, P.nt, P.pg,
                                                  P.np, h, r, th, ph, c);
}

// One segment of integrate_stokes_from_bricks_trace (accelerated_renderer.py:
// 113-125): the brick sampled at the midpoint of (p, q) (nothing outside the
// nonperiodic r / theta range), ds = L max(|q - p|, 1e-14), one RK2 or exact
// Stokes step and the optical depth.  Returns true once tau reaches the cutoff.
template <int Layout>
__device__ __forceinline__ bool transfer_segment(const BrickTraceParams &P, const AxisHints &h, const double p[3],
                                                 const double q[3], double S[4], double &tau, int &sampled) {
    double c[11];
    if (!sample_brick<Layout>(P, h, 0.5 * (p[0] + q[0]), 0.5 * (p[1] + q[1]), 0.5 * (p[2] + q[2]), c)) return false;
    const double dr = q[0] - p[0], dth = q[1] - p[1], dph = q[2] - p[2];
    const double dl = sqrt((dr * dr + dth * dth) + dph * dph);
    const double ds = fmax(P.length_cm * fmax(dl, 1.0e-14), 0.0);
    if (P.exact_step)
        stokes_step_exact(S, c, ds);
    else
        stokes_step_rk2_exact(S, c, ds);
    tau += fmax(c[4], 0.0) * ds;
    ++sampled;
    return tau >= P.max_tau;
}

// Four 128-thread blocks per SM (at most 128 registers): the 1024 x 576 image in 74.5 ms against
// 79.7 at three blocks and 95.4 unconstrained (248 registers), same image.
template <int Layout>
__global__ void __launch_bounds__(128, 4) brick_trace_kernel(const BrickTraceParams P) {
    const ViewDev &v = *P.view;
    const int64_t rays = (int64_t)v.crop_w * v.crop_h;
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ AxisHints shared_hints;  // the brick axes' first-guess parameters (the whole block)
    load_axis_hints(shared_hints, P.rg, P.nr, P.tg, P.nt, P.pg, P.np);
    const AxisHints hints = shared_hints;  // held in registers by the ray loop
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
            if (!stop_transfer && transfer_segment<Layout>(P, hints, y, yn, S, tau, sampled)) stop_transfer = true;
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

// ---------------------------------------------------------------- two-warp form
// For images with fewer warps than the GPU has schedulers (the reference's
// default 160 x 90 is 450 warps on 592), one warp per 32 rays leaves most of
// each scheduler idle while the warp waits on its own dependent FP64 chain:
// the RK4 steps and, for every step inside the brick, the sample and Stokes
// step.  Here a block of two warps takes 32 rays: warp 0 integrates the
// geodesics and publishes each accepted state through a ring of kRing slots in
// shared memory; warp 1 takes the segments from it -- sample, Stokes step,
// optical depth -- and reports the cutoff back.  Same arithmetic, same image.
constexpr int kRing = 32;
#ifndef BHN_PAIR_WARPS_PER_SM
#define BHN_PAIR_WARPS_PER_SM 4
#endif
constexpr int kPairWarpsPerSm = BHN_PAIR_WARPS_PER_SM;  // the two-warp form up to this many ray warps per SM
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s: a wait that long is a fault, not a delay
enum : int { kSlotDead = 0, kSlotLive = 1, kSlotEnd = 2 };

struct PairRing {
    double st[kRing][3][32];          // r, theta, phi after step j, at slot j % kRing
    int flag[kRing][32];              // kSlot*
    unsigned long long full[kRing];   // mbarriers: 32 arrivals (warp 0) per fill
    unsigned long long empty[kRing];  // 32 arrivals (warp 1) per drain
    int stop_step[32];                // warp 1 -> 0: step whose segment reached the cutoff (0: none)
    int end_steps[32], end_status[32];  // warp 0 -> 1, written before the end slot
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *b) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(b)) : "memory");
}
// Waits for the phase of parity `parity` to complete; false after kWaitCycles.
__device__ __forceinline__ bool mbar_wait(unsigned long long *b, unsigned parity) {
    const long long t0 = clock64();
    while (true) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(b)), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

template <int Layout>
__global__ void __launch_bounds__(64) brick_trace_pair_kernel(const BrickTraceParams P, unsigned *error_flags) {
    __shared__ PairRing R;
    __shared__ AxisHints shared_hints;
    const ViewDev &v = *P.view;
    const int64_t rays = (int64_t)v.crop_w * v.crop_h;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t r = (int64_t)blockIdx.x * 32 + lane;
    const bool in_image = r < rays;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kRing; ++k) {
            mbar_init(&R.full[k], 32);
            mbar_init(&R.empty[k], 32);
        }
    }
    if (threadIdx.x < 32) R.stop_step[threadIdx.x] = 0;
    load_axis_hints(shared_hints, P.rg, P.nr, P.tg, P.nt, P.pg, P.np);  // synchronises the block
    const int px = v.x0 + (int)(r % v.crop_w), py = v.y0 + (int)(r / v.crop_w);
    const bool traced = in_image && v.valid;

    if (warp == 0) {  // ------------------------------------------- geodesics
        double y[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, pt = 0.0, pphi = 0.0;
        const double a = v.a;
        if (traced) {
            const CameraRay cam = camera_ray(v, px, py);
            y[0] = v.r_obs;
            y[1] = v.theta_obs;
            y[2] = v.phi_obs;
            y[3] = cam.pr;
            y[4] = cam.pth;
            pt = cam.pt;
            pphi = cam.pphi;
        }
        const double r_edge = P.full_trace ? INFINITY : fmax(P.rg[0], P.rg[P.nr - 1]);
        bool alive = traced;
        int steps = 0, status = traced ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID;
        double prev_r = y[0];
        // slot j: the states after step j (j = 0: the camera), then one end slot
        auto publish = [&](int jj, int flag) -> bool {
            const int k = jj % kRing, f = jj / kRing;
            if (f > 0 && !__all_sync(0xffffffffu, mbar_wait(&R.empty[k], (f - 1) & 1))) return false;  // whole warp
            R.st[k][0][lane] = y[0];
            R.st[k][1][lane] = y[1];
            R.st[k][2][lane] = y[2];
            R.flag[k][lane] = flag;
            mbar_arrive(&R.full[k]);
            return true;
        };
        if (!publish(0, traced ? kSlotLive : kSlotDead)) {
            atomicOr(error_flags, 1u);
            return;
        }
        int i = 1;
        for (;; ++i) {
            // step i (kerr.py:355-378), while the transfer has not reached its cutoff
            const bool live = alive && i <= P.max_steps && *((volatile int *)&R.stop_step[lane]) == 0;
            if (!__any_sync(0xffffffffu, live)) break;
            int flag = kSlotDead;
            if (live) {
                double yn[5];
                rk4_state(y, P.step, a, pt, pphi, yn);
                steps = i;
                if (!(isfinite(yn[0]) && isfinite(yn[1]) && isfinite(yn[2]) && isfinite(yn[3]) && isfinite(yn[4]))) {
                    status = BHN_RAY_INVALID;  // kerr.py:364-366: the state is not stored
                    alive = false;
                } else {
                    for (int q = 0; q < 5; ++q) y[q] = yn[q];
                    flag = kSlotLive;
                    if (y[0] <= v.r_capture) {
                        status = BHN_RAY_CAPTURED;
                        alive = false;
                    } else if (y[0] > P.escape_radius && y[0] > prev_r) {
                        status = BHN_RAY_ESCAPED;
                        alive = false;
                    } else if (y[0] > r_edge && outbound_for_good(y[0], y[1], y[3], y[4], pt, pphi, a)) {
                        status = BHN_RAY_OUTBOUND;  // no later segment is sampled
                        alive = false;
                    }
                    prev_r = y[0];
                }
            }
            if (!publish(i, flag)) {
                atomicOr(error_flags, 1u);
                return;
            }
        }
        R.end_steps[lane] = steps;
        R.end_status[lane] = status;
        if (!publish(i, kSlotEnd)) atomicOr(error_flags, 1u);  // the end slot carries end_steps / end_status
    } else {  // ------------------------------------------------- transfer
        const AxisHints hints = shared_hints;
        double S[4] = {0.0, 0.0, 0.0, 0.0}, prev[3] = {0.0, 0.0, 0.0}, tau = 0.0;
        int sampled = 0, stop_at = 0;
        bool ok = true;
        for (int j = 0;; ++j) {
            const int k = j % kRing, f = j / kRing;
            if (!__all_sync(0xffffffffu, mbar_wait(&R.full[k], f & 1))) {  // the whole warp gives up together
                atomicOr(error_flags, 1u);
                ok = false;
                break;
            }
            const double cur[3] = {R.st[k][0][lane], R.st[k][1][lane], R.st[k][2][lane]};
            const int flag = R.flag[k][lane];
            mbar_arrive(&R.empty[k]);
            if (flag == kSlotEnd) break;
            if (flag == kSlotLive) {
                if (j > 0 && stop_at == 0 && transfer_segment<Layout>(P, hints, prev, cur, S, tau, sampled)) {
                    stop_at = j;  // the cutoff (accelerated_renderer.py:123-125): nothing later changes the image
                    R.stop_step[lane] = j;
                }
                prev[0] = cur[0];
                prev[1] = cur[1];
                prev[2] = cur[2];
            }
        }
        if (in_image) {
            const int64_t o = v.out_offset + r;
            for (int q = 0; q < 4; ++q) P.out[4 * o + q] = !ok ? NAN : (isfinite(S[q]) ? S[q] : 0.0);
            if (P.diag) {
                P.diag[4 * o + 0] = tau;
                P.diag[4 * o + 1] = sampled;
                P.diag[4 * o + 2] = stop_at ? stop_at : (ok ? R.end_steps[lane] : -1);
                P.diag[4 * o + 3] = stop_at ? BHN_RAY_OPAQUE : (ok ? R.end_status[lane] : -1);
            }
        }
    }
}

}  // namespace bhn

extern "C" int bhn_brick_trace_render(const void *coeffs, const double *r_grid, int32_t nr, const double *theta_grid,
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
    const int layout = cfg->coeff_layout;
    if (layout != BHN_BRICK_F64X11 && layout != BHN_BRICK_F32X12 && layout != BHN_BRICK_F64X12)
        return fail(BHN_ERR_VALUE, "unknown coefficient layout");
    if (layout != BHN_BRICK_F64X11 && (reinterpret_cast<uintptr_t>(coeffs) & 15u))
        return fail(BHN_ERR_VALUE, "cell records must be 16-byte aligned");
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
    // Two warps per 32 rays while the one-warp form would leave schedulers idle (at most one ray
    // warp per scheduler, 4 per SM); above that the one-warp form wins (200 x 112, 4.7 ray warps
    // per SM: 6.52 against 7.17 ms; 256 x 144, 7.8 per SM: even; 160 x 90, 3 per SM: 4.33 against 6.3).
    const int64_t warps = (rays + 31) / 32;
    if (warps <= (int64_t)kPairWarpsPerSm * sm_count_current_device()) {
        unsigned *flags = &reinterpret_cast<QueueState *>(static_cast<unsigned char *>(scratch) +
                                                          scratch_layout(1).queue)->error_flags;
        if (layout == BHN_BRICK_F32X12)
            brick_trace_pair_kernel<BHN_BRICK_F32X12><<<(unsigned)warps, 64, 0, as_stream(stream)>>>(P, flags);
        else if (layout == BHN_BRICK_F64X12)
            brick_trace_pair_kernel<BHN_BRICK_F64X12><<<(unsigned)warps, 64, 0, as_stream(stream)>>>(P, flags);
        else
            brick_trace_pair_kernel<BHN_BRICK_F64X11><<<(unsigned)warps, 64, 0, as_stream(stream)>>>(P, flags);
        BHN_LAUNCH_CHECK("brick_trace_pair_kernel");
        return BHN_OK;
    }
    const unsigned blocks = (unsigned)((rays + 127) / 128);
    if (layout == BHN_BRICK_F32X12)
        brick_trace_kernel<BHN_BRICK_F32X12><<<blocks, 128, 0, as_stream(stream)>>>(P);
    else if (layout == BHN_BRICK_F64X12)
        brick_trace_kernel<BHN_BRICK_F64X12><<<blocks, 128, 0, as_stream(stream)>>>(P);
    else
        brick_trace_kernel<BHN_BRICK_F64X11><<<blocks, 128, 0, as_stream(stream)>>>(P);
    BHN_LAUNCH_CHECK("brick_trace_kernel");
    return BHN_OK;
}
