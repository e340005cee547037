/*
 * blackhole_native.h -- C ABI of the B200 (sm_100a) GRRT hot-loop library
 * (libbhnative.so).
 *
 * Every entry point takes plain pointers and sizes.  Array arguments are
 * DEVICE pointers on the calling GPU unless a parameter name starts with h_;
 * `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 * asynchronous on `stream` unless stated otherwise.  Every function returns a
 * bhn_status; on failure bhn_last_error() holds a message (thread-local).
 *
 * The plugin micro-kernels replace the PyO3 functions of the reference's
 * native core (native/core/src/lib.rs) that python/blackhole_sim/
 * native_kernels.py binds; their float64 results reproduce the reference's
 * bit for bit.  Reference paths are relative to the reference project root.
 */
#ifndef BLACKHOLE_NATIVE_H
#define BLACKHOLE_NATIVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BHN_ABI_VERSION 1

typedef enum bhn_status {
    BHN_OK = 0,
    BHN_ERR_VALUE = 1,       /* bad argument; the message matches the reference's ValueError text */
    BHN_ERR_CUDA = 2,        /* CUDA runtime error */
    BHN_ERR_DEVICE = 3,      /* a kernel reported a failure through its status word */
    BHN_ERR_UNSUPPORTED = 4  /* not an sm_100 device, or a disabled feature */
} bhn_status;

/* Invalid-sample policies of native_kernels.py:15 / :342-350. */
enum { BHN_POLICY_NAN = 0, BHN_POLICY_INITIAL = 1, BHN_POLICY_ZERO = 2 };

/* Ray termination status (kerr.py:25 plus the optical-depth cutoff of
 * accelerated_renderer.py:123-125).  BHN_RAY_OUTBOUND (brick and GRRT renderers):
 * the ray is past the brick's (or snapshot's) outer radius, moving out, and
 * can never turn back, so no later segment is sampled and its image is final. */
enum {
    BHN_RAY_MAX_STEPS = 0,
    BHN_RAY_CAPTURED = 1,
    BHN_RAY_ESCAPED = 2,
    BHN_RAY_INVALID = 3,
    BHN_RAY_OPAQUE = 4,
    BHN_RAY_OUTBOUND = 5
};

/* ---- library ------------------------------------------------------------ */

/* Replaces core_version() (native/core/src/lib.rs:19-22). */
const char *bhn_core_version(void);
/* Message of the last failure on this host thread ("" if none). */
const char *bhn_last_error(void);
/* Device properties of the current device (detect_arch() of lib.rs:24-35 is
 * answered by the host binding; this reports the GPU side). */
int bhn_device_info(int32_t *sm_count, int32_t *cc_major, int32_t *cc_minor, int64_t *global_mem_bytes);

/* FP32 FMA throughput probe used as the denominator of the FP32 roofline (no
 * reference counterpart: a measurement aid).  Launches SMs * blocks_per_sm
 * blocks of 256 threads doing iters * 128 FMAs each; *flops receives the FLOP
 * count (2 per FMA).  scratch: >= SMs * blocks_per_sm * 256 floats (never
 * written in practice). */
int bhn_fp32_peak_probe(float *scratch, int32_t iters, int32_t blocks_per_sm, int64_t *flops, void *stream);

/* FP64 throughput probe, the denominator of the synchrotron kernels' rooflines
 * (a measurement aid like the FP32 probe).  mode 0: iters * 128 FP64 FMAs per
 * thread, *ops = FLOP (2 per FMA); mode 1: iters * 32 double-precision exp()
 * calls per thread in 8 independent chains, *ops = exp evaluations.  Same
 * launch shape and scratch size (doubles) as bhn_fp32_peak_probe. */
int bhn_fp64_peak_probe(double *scratch, int32_t iters, int32_t blocks_per_sm, int32_t mode, int64_t *ops,
                        void *stream);

/* ---- plugin micro-kernels (float64, bit-exact with the reference) -------- */

/* Replaces stokes_rk2_brick (native/core/src/lib.rs:227-279).  coeffs: cells*11,
 * initial: 4 (broadcast) or 4*cells values, out: 4*cells. */
int bhn_stokes_rk2_brick(const double *coeffs, int64_t cells, double ds_cm, const double *initial,
                         int64_t initial_len, double *out, void *stream);

/* The exact constant-coefficient Stokes step of
 * python/blackhole_sim/polarized_transfer.py:51-70 (stokes_step_exact: the
 * 5x5 augmented exponential exp([[-K, j], [0, 0]] ds) applied to [S; 1]) for
 * every cell, with the input contract of bhn_stokes_rk2_brick.  The reference
 * evaluates it one step at a time through scipy.linalg.expm; here by scaling
 * and squaring with a truncated Taylor series in FP64. */
int bhn_stokes_exact_brick(const double *coeffs, int64_t cells, double ds_cm, const double *initial,
                           int64_t initial_len, double *out, void *stream);

/* Replaces sample_brick_trilinear (native/core/src/lib.rs:281-306).  coeffs:
 * nr*nt*np*11 in [r][theta][phi][11] order, points: n*3 (r, theta, phi),
 * out: n*11 with NaN rows outside the nonperiodic r/theta domain. */
int bhn_sample_brick_trilinear(const double *coeffs, const double *r_grid, int64_t nr, const double *theta_grid,
                               int64_t nt, const double *phi_grid, int64_t np, const double *points,
                               int64_t n_points, double *out, void *stream);

/* Replaces sample_and_step_stokes (native/core/src/lib.rs:308-366) and, for a
 * policy other than BHN_POLICY_NAN, also the Python-side policy overwrite of
 * native_kernels.py:391-397.  out: n*4. */
int bhn_sample_and_step_stokes(const double *coeffs, const double *r_grid, int64_t nr, const double *theta_grid,
                               int64_t nt, const double *phi_grid, int64_t np, const double *points,
                               int64_t n_points, double ds_cm, const double *initial, int64_t initial_len,
                               int32_t invalid_policy, double *out, void *stream);

/* bhn_sample_and_step_stokes with the points taken in brick-cell order: a
 * key kernel brackets every point (cell index, or past-the-end for points
 * outside the nonperiodic r/theta domain), a radix sort orders the point
 * indices by cell, and the sampler walks that order, writing each result to
 * its point's own row -- the same values, bit for bit, with neighbouring
 * points sharing cached corners.  For 0 < n_points < 2^31 and cells < 2^32 - 1;
 * scratch: bhn_sample_sort_scratch_bytes(n_points, nr * nt * np) bytes,
 * 256-byte aligned, on the device. */
int64_t bhn_sample_sort_scratch_bytes(int64_t n_points, int64_t cells);
/* bhn_sample_brick_trilinear in the same cell order (same values, same scratch). */
int bhn_sample_brick_trilinear_sorted(const double *coeffs, const double *r_grid, int64_t nr, const double *theta_grid,
                                      int64_t nt, const double *phi_grid, int64_t np, const double *points,
                                      int64_t n_points, double *out, void *scratch, int64_t scratch_bytes,
                                      void *stream);
int bhn_sample_and_step_stokes_sorted(const double *coeffs, const double *r_grid, int64_t nr,
                                      const double *theta_grid, int64_t nt, const double *phi_grid, int64_t np,
                                      const double *points, int64_t n_points, double ds_cm, const double *initial,
                                      int64_t initial_len, int32_t invalid_policy, double *out, void *scratch,
                                      int64_t scratch_bytes, void *stream);

/* Replaces sample_brick_valid_mask (native_kernels.py:189-210, Python-only in
 * the reference): inclusive r/theta bounds, phi ignored.  mask: n bytes (0/1). */
int bhn_sample_brick_valid_mask(const double *r_grid, int64_t nr, const double *theta_grid, int64_t nt,
                                const double *points, int64_t n_points, uint8_t *mask, void *stream);

/* Input checks of native/core/src/lib.rs:112-169 on device data: counts[0] +=
 * number of non-finite values; counts[1] += number of i with values[i+1] <=
 * values[i] when check_increasing != 0.  counts: 2 device uint32 (zeroed by
 * the caller). */
int bhn_check_values(const double *values, int64_t n, int32_t check_increasing, uint32_t *counts, void *stream);

/* ---- coefficient bricks for the fused renderer ---------------------------- */

/* Record layout: one cell = 12 values (the 11 COEFF_NAMES channels of
 * python/blackhole_sim/coefficient_bricks.py:21-25 plus one pad), float32
 * records are 3 float4 (48 B), float64 records 6 double2 (96 B). */
#define BHN_RECORD_VALUES 12

/* Bytes of the grid-table buffer for an nr x nt x np brick. */
int64_t bhn_brick_tables_bytes(int32_t nr, int32_t nt, int32_t np);

/* Builds the lookup tables (grids, reciprocal spacings, closed-form index
 * parameters) from the three strictly increasing float64 grids. */
int bhn_brick_build_tables(const double *r_grid, int32_t nr, const double *theta_grid, int32_t nt,
                           const double *phi_grid, int32_t np, void *tables, void *stream);

/* Repacks [cells][11] coefficients (coeff_bytes 4 = float32, 8 = float64) into
 * records of record_bytes 4 (float32) or 8 (float64); nonfinite[0] += number
 * of non-finite inputs (device uint32, zeroed by the caller). */
int bhn_brick_pack(const void *coeffs, int32_t coeff_bytes, int64_t cells, void *records, int32_t record_bytes,
                   uint32_t *nonfinite, void *stream);

/* Cell location used by the fused renderer, exposed for bit-exact checks:
 * index[4*i..] = (i_r0, i_theta0, i_phi0, valid), weights[3*i..] = (w_r, w_theta,
 * w_phi) as float.  Indices equal numpy.searchsorted(side="right") - 1 with
 * the clamps of native_kernels.py:137-161. */
int bhn_brick_locate(const void *tables, int32_t nr, int32_t nt, int32_t np, const double *points, int64_t n_points,
                     int32_t *index, float *weights, void *stream);

/* ---- fused ray renderer ----------------------------------------------------- */

/* One camera view (kerr.py:155-233 LocalCamera, accelerated_renderer.py:36-46).
 * Angles in radians except fov_y_deg / roll_deg.  The step is
 * h = clamp(h_scale * r, h_min, h_max).  The view renders the rectangle
 * [x0, x0+crop_w) x [y0, y0+crop_h) of a width x height image; its pixels are
 * written row-major at out + out_offset. */
typedef struct bhn_view {
    double spin_a;
    double r_obs, theta_obs, phi_obs;
    double fov_y_deg, roll_deg;
    double h_scale, h_min, h_max;
    double escape_radius;
    double affine_to_length_cm;
    double max_optical_depth;
    int32_t width, height;
    int32_t x0, y0, crop_w, crop_h;
    int32_t max_steps;
    int32_t flags;           /* BHN_VIEW_* bits */
    int64_t out_offset;
} bhn_view;

/* Horizon guard (no reference counterpart; off = the reference's semantics):
 * a ray moving inward (p_r < 0) from inside both the innermost photon orbit
 * (the prograde equatorial circular photon orbit, inside which no ray from the
 * camera can turn around) and the brick's inner radius is captured at that
 * step.  In exact arithmetic no further emission can be added, so the image is
 * unchanged; numerically it stops the h = 0.02 r RK2 step from overshooting
 * into the horizon region, where it can fling a ray back through the brick. */
#define BHN_VIEW_HORIZON_GUARD 1

/* Launch shape, chosen by the autotuner. */
typedef struct bhn_render_config {
    int32_t block_threads;   /* 64..512, multiple of 32 */
    int32_t blocks_per_sm;   /* persistent grid = SM count * blocks_per_sm */
    int32_t tile_w, tile_h;  /* ray order: rays of one tile are consecutive in the queue */
    int32_t refill_min;      /* a warp refills its dead lanes once this many (1..32) are dead */
    int32_t precision;       /* 0 = FP32 fused kernel, 1 = FP64 (oracle-matched) kernel */
    int32_t reg_cap;         /* FP32 kernel register budget: 0 (compiler's choice), 80 or 64 */
} bhn_render_config;

/* Launch totals accumulated on the device (all zeroed by each launch). */
typedef struct bhn_render_stats {
    unsigned long long ray_steps;      /* geodesic RK2 steps executed by live rays */
    unsigned long long brick_steps;    /* steps whose midpoint sample was inside the brick */
    unsigned long long rays;           /* rays traced */
    unsigned long long status[5];      /* rays per BHN_RAY_* */
    unsigned long long queue_fetches;  /* work-queue atomics issued */
    float max_h_drift;                 /* max over rays of max |H - H0| (kerr.py:352, 367) */
    uint32_t error_flags;              /* nonzero: a kernel detected an inconsistency */
    float max_h_drift_escaped;         /* the same over escaped rays only (a captured ray's last
                                          state sits at the horizon, where H is ill-conditioned) */
    uint32_t pad0;
} bhn_render_stats;

/* Optional per-ray outputs (any pointer may be NULL), indexed like the image. */
typedef struct bhn_ray_outputs {
    int32_t *steps;
    uint8_t *status;
    float *h_drift;
} bhn_ray_outputs;

/* Bytes of device scratch a render over n_views views needs (work-queue head,
 * per-view tables, launch totals). */
int64_t bhn_render_scratch_bytes(int32_t n_views);

/* Uploads and derives the per-view tables into scratch (h_views is host memory,
 * copied before return).  Call again when the views change. */
int bhn_render_prepare(const bhn_view *h_views, int32_t n_views, void *scratch, int64_t scratch_bytes,
                       void *stream);

/* Runs the fused persistent kernel over all prepared views: camera ray (FP64)
 * -> RK2 Kerr geodesic -> midpoint brick gather -> Stokes RK2 -> optical-depth
 * cutoff, per accelerated_renderer.py:100-150 and kerr.py:337-384.  records is
 * float32 (precision 0) or float64 (precision 1) records; out is float4
 * (precision 0) or double4 (precision 1) Stokes (I, Q, U, V) per pixel; stats
 * (device, may be NULL) receives the launch totals. */
int bhn_render_launch(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                      const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                      int64_t scratch_bytes, bhn_render_stats *stats, void *stream);

/* bhn_render_prepare + bhn_render_launch for callers that cannot allocate
 * device memory (no counterpart in the reference).  Some hosts own all device
 * memory through their own allocator or a pool sized at start-up, and a
 * library they load may not allocate beside it; real-time loops may not take
 * the device-wide synchronisation that cudaMalloc / cudaFree can imply.  Such
 * callers pass only inputs and outputs.  The scratch is a fixed 64 KiB array
 * in the library's device image (held by every GPU that loads the library
 * until the process exits), so at most BHN_NOALLOC_MAX_VIEWS views fit in one
 * call; more is rejected with BHN_ERR_VALUE.  The first call on a device does
 * the set-up: it looks up that array's device address (cudaGetSymbolAddress)
 * with the device current and keeps it for the process, so make the first
 * call on each device before any stream capture, and do not call it after
 * cudaDeviceReset.  All calls on a device share the array and each call
 * rewrites the part it uses (the work-queue head and the launch totals are
 * zeroed by every launch): calls that overlap on the GPU (different streams,
 * or the same stream from several host threads without ordering) race.  The
 * function allocates nothing (no cudaMalloc / cudaFree, no library allocator);
 * h_views is ordinary host memory, copied into the array before the call
 * returns; stats may be NULL. */
#define BHN_NOALLOC_MAX_VIEWS 120
int bhn_render_noalloc(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np,
                       const bhn_view *h_views, int32_t n_views, const bhn_render_config *cfg, void *out,
                       const bhn_ray_outputs *ray_out, bhn_render_stats *stats, void *stream);

/* ---- learned step-size proposal (no reference counterpart) ----
 * The plain method is kerr.py:337-384's loop with the RK2 step of
 * native/cuda/kerr_stokes_kernel.cu:13 at h = clamp(h_scale r, h_min, h_max).
 * These entry points add (1) an RK2 step-doubling controller that renders the
 * adaptive image and records training samples, (2) training kernels for an
 * 8 -> 64 -> 64 -> 1 SiLU network (BF16 weights, FP32 accumulation) that maps
 * the ray state to log h, and (3) the ray loop that takes the network's step
 * and falls back to the plain step when an embedded error check fails.  All
 * three always apply BHN_VIEW_HORIZON_GUARD. */
typedef struct bhn_adapt_params {
    float tol;           /* mixed-norm tolerance: |e_i| <= tol (1 + |y_i|) over r, theta, phi, p_r, p_theta */
    float sample_prob;   /* controller: probability of recording an accepted step */
    float h_floor, h_ceil;
    float margin;        /* learned: subtracted from the network's log multiplier of the plain step */
    float check_tol;     /* learned: tolerance of the embedded Euler-midpoint check h|k2 - k1| (0: none) */
    float brick_scale;   /* both: inside the brick's (r, theta) box the step is at most brick_scale times the
                            plain step clamp(h_scale r, h_min, h_max), and a step entering the box ends at most
                            one such step past the entry point (0: no limit) */
    float min_scale;     /* learned: the step is at least min_scale times the plain step (> 0) */
    int32_t interval;    /* learned: steps between network evaluations (the multiplier is kept in between) */
    int32_t max_attempts; /* controller: attempts per step before the step is forced */
    int32_t fallback;    /* learned: a step failing the check is the plain step (0), the controller's (1), or
                            retried by the lane with a shorter proposal next iteration (2; at most max_attempts) */
    uint32_t seed;       /* controller: sample-selection hash seed */
    int32_t substeps;    /* learned: 1 = one RK2 step of the proposed h per brick segment; 2 = two RK2 steps of
                            h / 2 per segment (the controller's accepted-solution form, without its h-step
                            error estimate), each half step checked */
} bhn_adapt_params;

/* Sample rows: 8 raw features (log r, cos theta, asinh p_r, asinh p_theta, a,
 * log|Delta|, p_phi, log(j_I + 1e-12)) followed by log(h_opt / h_plain):
 * h_opt = h err^(-1/3) is the step at which the controller's error estimate
 * equals the tolerance, h_plain = clamp(h_scale r, h_min, h_max) the plain
 * step at the same r (9 floats). */
#define BHN_SAMPLE_FLOATS 9
int64_t bhn_mlp_param_count(void);
int64_t bhn_mlp_blob_bytes(void);
/* FP32 parameters [W1 8x64 | b1 | W2 64x64 | b2 | W3 64 | b3] (device) +
 * h_norm (host: mu_x[8], 1/sigma_x[8], mu_y, sigma_y) -> inference blob (BF16
 * fragments, device). */
int bhn_mlp_pack(const float *params, const float *h_norm, void *blob, void *stream);
/* grad += d(mean squared error)/d(params) over rows index[first .. first+count)
 * of standardised samples; loss += sum of squared errors. */
int bhn_mlp_grad(const float *params, const float *samples, const int64_t *index, int64_t first, int64_t count,
                 float *grad, float *loss, void *stream);
/* One Adam step (step counts from 1); clears grad. */
int bhn_mlp_adam(float *params, float *grad, float *m, float *v, float lr, float beta1, float beta2, float eps,
                 int32_t step, void *stream);
/* The inference path on given standardised feature rows (n x 8) -> n outputs. */
int bhn_mlp_infer(const void *blob, const float *features, int64_t n, float *out, void *stream);
/* Step-doubling controller over prepared views (bhn_render_prepare): float4
 * Stokes out, optional per-ray steps/status/Hamiltonian drift, samples appended while
 * *sample_count < capacity; counters[0..2] += RK2 stage pairs, accepted steps,
 * rejected attempts. */
int bhn_adaptive_launch(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                        const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                        int64_t scratch_bytes, const bhn_adapt_params *params, float *samples,
                        unsigned long long *sample_count, unsigned long long sample_capacity,
                        unsigned long long *counters, void *stream);
/* The learned-step ray loop over prepared views (optional per-ray
 * steps/status/Hamiltonian drift); counters[0..3] += RHS evaluations, steps,
 * fallbacks, network evaluations. */
int bhn_learned_launch(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                       const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                       int64_t scratch_bytes, const bhn_adapt_params *params, const void *blob,
                       unsigned long long *counters, void *stream);

/* ---- coefficient-brick precompute --------------------------------------------
 * Replaces precompute_coefficient_bricks (python/blackhole_sim/
 * coefficient_bricks.py:119-152) with the Hybrid synchrotron model
 * (python/blackhole_sim/synchrotron.py:240-325): per cell the local plasma frame
 * of coefficient_bricks.py:110-116 (n_e = rho * rho_cgs_per_code / (mu_e m_p),
 * B = |b_con[1:4]| * b_gauss_per_code, EVPA = atan2(b^3, b^2), Theta_e floored
 * at 1e-8, no line-of-sight pitch), then the thermal and power-law
 * components' 11 coefficients, summed, rotated by the EVPA and written in
 * COEFF_NAMES order with the brick dtype's nan_to_num.  FP64 throughout. */
typedef struct bhn_synchrotron_model {
    double nu_hz;
    double rho_cgs_per_code, b_gauss_per_code, mean_molecular_weight_per_electron;  /* PhysicalScaling */
    int32_t thermal, nonthermal;                   /* which components the model sums (Hybrid: both) */
    int32_t thermal_gamma_n, thermal_pitch_n;      /* ThermalSynchrotronCoefficients: 192, 16 */
    double thermal_rotation_scale, thermal_conversion_scale;                 /* 1, 1 */
    int32_t nonthermal_gamma_n, nonthermal_pitch_n;                          /* 224, 16 */
    double nonthermal_p, nonthermal_gamma_min, nonthermal_gamma_max;         /* 3.5, 10, 1e5 */
    double nonthermal_fraction, nonthermal_absorption_scale, nonthermal_faraday_scale;  /* 0.02, 1, 0.15 */
} bhn_synchrotron_model;

/* rho, theta_e: [cells] float64 (device); b_con: [cells][4] float64 (device);
 * coeffs: [cells][11] of coeff_bytes (4 or 8) each (device).  Gamma grids take
 * 2..4096 nodes, pitch averages 1..64. */
int bhn_brick_precompute(const double *rho, const double *theta_e, const double *b_con, int64_t cells,
                         const bhn_synchrotron_model *model, void *coeffs, int32_t coeff_bytes, void *stream);

/* The model's 11 coefficients for n local plasma frames, FP64 on the device.
 * Replaces ThermalSynchrotronCoefficients.coefficients,
 * NonthermalPowerLawSynchrotronCoefficients.coefficients and
 * HybridSynchrotronCoefficients.coefficients (python/blackhole_sim/
 * synchrotron.py:248, 290, 318), per frame of synchrotron.py:28-44:
 * frames[n][5] = (n_e_cm3, theta_e, b_gauss, cos_pitch_to_los, evpa_rad)
 * (device), out[n][11] in PolarizedCoefficients field order, which is
 * COEFF_NAMES order (device).  No nan_to_num, no Theta_e floor beyond the
 * models' own; the scaling fields of the model are not used. */
int bhn_synchrotron_coefficients(const double *frames, int64_t n, const bhn_synchrotron_model *model, double *out,
                                 void *stream);

/* ---- physical polarized GRRT through a GRMHD snapshot --------------------------
 * Replaces polarized_renderer.render_stokes_image (python/blackhole_sim/
 * polarized_renderer.py:31-70): per pixel of one view, the camera ray
 * (kerr.py:188-233), a fixed-step RK4 geodesic (kerr.py:306-313, 337-384) and
 * integrate_polarized_kerr_grrt (polarized_transfer.py:83-145) with the
 * synchrotron model of bhn_brick_precompute, in FP64.  fields:
 * [nr][nt][np][11] float64 = rho, Theta_e, pressure, b^mu (4), u^mu (4) of the
 * snapshot (grmhd.py:55-121); out: [rays][4] Stokes of the view's crop in row
 * order (at view->out_offset); diag (optional): [rays][8] = optical depth,
 * emitting segments, valid segments, Faraday depth, min / max redshift,
 * steps traced, BHN_RAY_* status.  scratch: bhn_grrt_scratch_bytes(rays,
 * chunk) bytes, 256-byte aligned; the renderer lists up to `chunk` emitting
 * segments per ray and round (the largest chunk the scratch holds, <= 4096),
 * so a larger scratch means fewer rounds.  Results do not depend on it. */
typedef struct bhn_grrt_config {
    double step;                 /* affine RK4 step (PolarizedRenderConfig.step) */
    double escape_radius;
    double nu_hz;                /* observing frequency */
    double length_cm;            /* affine-to-length scale (the scaling's r_g when not given) */
    double max_optical_depth, min_redshift, flux_scale;
    int32_t max_steps;
    int32_t exact_step;          /* 1: stokes_step_exact, 0: RK2 (PolarizedTransferConfig.use_exact_matrix_step) */
    int32_t full_trace;          /* 1: trace every ray to the reference's own end; 0: also end a ray past the
                                    snapshot's outer radius moving out for good (BHN_RAY_OUTBOUND, same image) */
} bhn_grrt_config;
int64_t bhn_grrt_scratch_bytes(int64_t rays, int32_t chunk);
int bhn_grrt_render(const double *fields, const double *r_grid, int32_t nr, const double *theta_grid, int32_t nt,
                    const double *phi_grid, int32_t np, const bhn_view *view, const bhn_synchrotron_model *model,
                    const bhn_grrt_config *cfg, void *scratch, int64_t scratch_bytes, double *out, double *diag,
                    void *stream);

/* ---- the reference's brick renderer (RK4 fixed step) ----------------------
 * Replaces render_stokes_image_bricks / render_tile_stokes_bricks
 * (python/blackhole_sim/accelerated_renderer.py:100-158): per pixel of one
 * view (a crop = a tile) the camera ray, a fixed-step RK4 geodesic
 * (kerr.py:306-313, 337-384) and integrate_stokes_from_bricks_trace: the
 * coefficient brick sampled at each segment's midpoint (no sample outside the
 * nonperiodic r / theta range), ds = length_cm * max(|d(r, theta, phi)|,
 * 1e-14), an RK2 or exact Stokes step, the optical-depth cutoff, and
 * non-finite results set to 0; FP64, one thread per ray.  (bhn_render_launch
 * is the RK2, h = 0.02 r form of the same loop.)  coeffs: per
 * cfg->coeff_layout, [nr][nt][np][11] float64 (BHN_BRICK_F64X11, the
 * CoefficientBrickGrid layout) or [nr][nt][np][12] cell records, 11 channels
 * and one unused pad, 16-byte aligned, in float32 (BHN_BRICK_F32X12: a float32
 * brick, read with three 128-bit loads per cell) or float64
 * (BHN_BRICK_F64X12); the interpolation is float64 either way (float32 values
 * widen exactly), so the three give the same image; out: [rays][4] at view->out_offset; diag (optional): [rays][4] =
 * optical depth, sampled segments, RK4 steps taken, BHN_RAY_* status.
 * Unless full_trace is set, a ray's trace also ends once it is past the
 * brick's outer radius, moving out, with a radial potential that keeps it
 * moving out (R(r') >= E^2 r'^4 / 4 for every r' beyond it: status
 * BHN_RAY_OUTBOUND): no later segment can be sampled, so the image is the
 * same bit for bit, and only the diag columns "RK4 steps taken" and
 * "status" differ from the full trace's.
 * scratch: bhn_render_scratch_bytes(1). */
enum { BHN_BRICK_F64X11 = 0, BHN_BRICK_F32X12 = 1, BHN_BRICK_F64X12 = 2 };
typedef struct bhn_brick_trace_config {
    double step;                 /* affine RK4 step (AcceleratedRenderConfig.step) */
    double escape_radius;
    double length_cm;            /* affine_to_length_cm (1.0 when the config leaves it unset) */
    double max_optical_depth;
    int32_t max_steps;
    int32_t exact_step;          /* 1: stokes_step_exact, 0: RK2 */
    int32_t full_trace;          /* 1: trace every ray to the reference's own end (escape radius, capture,
                                    max_steps), 0: also end outbound rays past the brick (same image) */
    int32_t coeff_layout;        /* BHN_BRICK_*: layout of coeffs */
} bhn_brick_trace_config;
int bhn_brick_trace_render(const void *coeffs, const double *r_grid, int32_t nr, const double *theta_grid,
                           int32_t nt, const double *phi_grid, int32_t np, const bhn_view *view,
                           const bhn_brick_trace_config *cfg, void *scratch, int64_t scratch_bytes, double *out,
                           double *diag, void *stream);

/* CUDA-graph form of bhn_render_launch: captures the queue reset and the
 * persistent launch once; bhn_graph_launch replays it on `stream`. */
typedef struct bhn_graph bhn_graph;
int bhn_graph_create(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                     const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                     int64_t scratch_bytes, bhn_render_stats *stats, bhn_graph **graph);
int bhn_graph_launch(bhn_graph *graph, void *stream);
int bhn_graph_destroy(bhn_graph *graph);

#ifdef __cplusplus
}
#endif

#endif /* BLACKHOLE_NATIVE_H */
