// bhn_api.cu -- library plumbing, float64 plugin micro-kernels, brick tables.
//
// The micro-kernels reproduce the reference's float64 arithmetic operation by
// operation: every multiply, add and subtract goes through the explicit
// round-to-nearest intrinsics (__dmul_rn / __dadd_rn / __dsub_rn), which the
// compiler never contracts into FMAs, and divisions / fmod are IEEE exact on
// the GPU.  Results therefore equal numpy's (native_kernels.py) and the Rust
// core's (native/core/src/lib.rs) bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "bhn_internal.cuh"
#include "bhn_transfer.cuh"
#include "bhn_exact.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace bhn {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t err, const char *what) {
    g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(err);
    return BHN_ERR_CUDA;
}

int sm_count_current_device() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cached[dev] == 0) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        cached[dev] = sms;
    }
    return cached[dev];
}

// exact helpers: bhn_exact.cuh

// ------------------------------------------------------------------- kernels
__global__ void stokes_rk2_brick_kernel(const double *__restrict__ coeffs, int64_t cells, double ds,
                                        const double *__restrict__ initial, int broadcast, double *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cells; i += (int64_t)gridDim.x * blockDim.x) {
        double c[11];
#pragma unroll
        for (int k = 0; k < 11; ++k) c[k] = coeffs[11 * i + k];
        const double *s0 = initial + (broadcast ? 0 : 4 * i);
        double s[4] = {s0[0], s0[1], s0[2], s0[3]};
        stokes_step_rk2_exact(s, c, ds);
        reinterpret_cast<double2 *>(out + 4 * i)[0] = make_double2(s[0], s[1]);
        reinterpret_cast<double2 *>(out + 4 * i)[1] = make_double2(s[2], s[3]);
    }
}

__global__ void stokes_exact_brick_kernel(const double *__restrict__ coeffs, int64_t cells, double ds,
                                          const double *__restrict__ initial, int broadcast, double *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cells; i += (int64_t)gridDim.x * blockDim.x) {
        double c[11];
#pragma unroll
        for (int k = 0; k < 11; ++k) c[k] = coeffs[11 * i + k];
        const double *s0 = initial + (broadcast ? 0 : 4 * i);
        double s[4] = {s0[0], s0[1], s0[2], s0[3]};
        stokes_step_exact(s, c, ds);
        reinterpret_cast<double2 *>(out + 4 * i)[0] = make_double2(s[0], s[1]);
        reinterpret_cast<double2 *>(out + 4 * i)[1] = make_double2(s[2], s[3]);
    }
}

__device__ __forceinline__ void sample_trilinear_point(const double *__restrict__ coeffs, const double *__restrict__ rg,
                                                       int nr, const double *__restrict__ tg, int nt,
                                                       const double *__restrict__ pg, int np,
                                                       const double *__restrict__ pts, int64_t i,
                                                       double *__restrict__ out) {
    double c[11];
    if (!sample_one_exact(coeffs, rg, nr, tg, nt, pg, np, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], c)) {
#pragma unroll
        for (int k = 0; k < 11; ++k) c[k] = __longlong_as_double(0x7ff8000000000000ULL);
    }
#pragma unroll
    for (int k = 0; k < 11; ++k) out[11 * i + k] = c[k];
}

__global__ void sample_trilinear_kernel(const double *__restrict__ coeffs, const double *__restrict__ rg, int nr,
                                        const double *__restrict__ tg, int nt, const double *__restrict__ pg, int np,
                                        const double *__restrict__ pts, int64_t n, double *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        sample_trilinear_point(coeffs, rg, nr, tg, nt, pg, np, pts, i, out);
}

__global__ void sample_trilinear_ordered_kernel(const double *__restrict__ coeffs, const double *__restrict__ rg,
                                                int nr, const double *__restrict__ tg, int nt,
                                                const double *__restrict__ pg, int np, const double *__restrict__ pts,
                                                const uint32_t *__restrict__ order, int64_t n,
                                                double *__restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        sample_trilinear_point(coeffs, rg, nr, tg, nt, pg, np, pts, (int64_t)order[k], out);
}

__global__ void sample_and_step_kernel(const double *__restrict__ coeffs, const double *__restrict__ rg, int nr,
                                       const double *__restrict__ tg, int nt, const double *__restrict__ pg, int np,
                                       const double *__restrict__ pts, int64_t n, double ds,
                                       const double *__restrict__ initial, int broadcast, int policy,
                                       double *__restrict__ out);

// One Stokes RK2 sample-and-step of point i (native_kernels.py:325-407 with the policy of :391-397).
__device__ __forceinline__ void sample_and_step_point(const double *__restrict__ coeffs, const double *__restrict__ rg,
                                                      int nr, const double *__restrict__ tg, int nt,
                                                      const double *__restrict__ pg, int np,
                                                      const double *__restrict__ pts, int64_t i, double ds,
                                                      const double *__restrict__ initial, int broadcast, int policy,
                                                      double *__restrict__ out) {
    double c[11];
    const double *s0 = initial + (broadcast ? 0 : 4 * i);
    double s[4] = {s0[0], s0[1], s0[2], s0[3]};
    if (sample_one_exact(coeffs, rg, nr, tg, nt, pg, np, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], c)) {
        stokes_step_rk2_exact(s, c, ds);
    } else if (policy == BHN_POLICY_ZERO) {
        s[0] = s[1] = s[2] = s[3] = 0.0;
    } else if (policy != BHN_POLICY_INITIAL) {
        s[0] = s[1] = s[2] = s[3] = __longlong_as_double(0x7ff8000000000000ULL);
    }
    reinterpret_cast<double2 *>(out + 4 * i)[0] = make_double2(s[0], s[1]);
    reinterpret_cast<double2 *>(out + 4 * i)[1] = make_double2(s[2], s[3]);
}

// The cell (r0, theta0, phi0) a point samples from, as one index; points the
// sampler rejects (outside the nonperiodic r/theta range, non-finite) sort last.
__global__ void cell_key_kernel(const double *__restrict__ rg, int nr, const double *__restrict__ tg, int nt,
                                const double *__restrict__ pg, int np, const double *__restrict__ pts, int64_t n,
                                uint32_t invalid_key, uint32_t *__restrict__ keys, uint32_t *__restrict__ idx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int r0, t0, p0, p1;
        double wr, wt, wp;
        uint32_t key = invalid_key;
        if (bracket_linear_exact(rg, nr, pts[3 * i], r0, wr) && bracket_linear_exact(tg, nt, pts[3 * i + 1], t0, wt)) {
            bracket_phi_exact(pg, np, pts[3 * i + 2], p0, p1, wp);
            key = (uint32_t)(((int64_t)r0 * nt + t0) * np + p0);
        }
        keys[i] = key;
        idx[i] = (uint32_t)i;
    }
}

__global__ void sample_and_step_kernel(const double *__restrict__ coeffs, const double *__restrict__ rg, int nr,
                                       const double *__restrict__ tg, int nt, const double *__restrict__ pg, int np,
                                       const double *__restrict__ pts, int64_t n, double ds,
                                       const double *__restrict__ initial, int broadcast, int policy,
                                       double *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        sample_and_step_point(coeffs, rg, nr, tg, nt, pg, np, pts, i, ds, initial, broadcast, policy, out);
}

__global__ void sample_and_step_ordered_kernel(const double *__restrict__ coeffs, const double *__restrict__ rg,
                                               int nr, const double *__restrict__ tg, int nt,
                                               const double *__restrict__ pg, int np, const double *__restrict__ pts,
                                               const uint32_t *__restrict__ order, int64_t n, double ds,
                                               const double *__restrict__ initial, int broadcast, int policy,
                                               double *__restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        sample_and_step_point(coeffs, rg, nr, tg, nt, pg, np, pts, (int64_t)order[k], ds, initial, broadcast, policy,
                              out);
}

__global__ void valid_mask_kernel(const double *__restrict__ rg, int nr, const double *__restrict__ tg, int nt,
                                  const double *__restrict__ pts, int64_t n, uint8_t *__restrict__ mask) {
    const double r0 = rg[0], rN = rg[nr - 1], t0 = tg[0], tN = tg[nt - 1];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double r = pts[3 * i], th = pts[3 * i + 1];
        mask[i] = (uint8_t)((r >= r0) & (r <= rN) & (th >= t0) & (th <= tN));
    }
}

__global__ void check_values_kernel(const double *__restrict__ v, int64_t n, int check_inc, uint32_t *counts) {
    uint32_t bad = 0, nonmono = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = v[i];
        bad += !isfinite(x);
        if (check_inc && i + 1 < n) nonmono += !(v[i + 1] > x);
    }
    for (int o = 16; o > 0; o >>= 1) {
        bad += __shfl_down_sync(0xffffffffu, bad, o);
        nonmono += __shfl_down_sync(0xffffffffu, nonmono, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (bad) atomicAdd(counts, bad);
        if (nonmono) atomicAdd(counts + 1, nonmono);
    }
}

// Grid tables: one block, thread 0..2 classify an axis each.
__global__ void build_tables_kernel(const double *__restrict__ rg, int nr, const double *__restrict__ tg, int nt,
                                    const double *__restrict__ pg, int np, void *tables) {
    Tables T = tables_at(tables, nr, nt, np);
    TableHeader *h = const_cast<TableHeader *>(T.h);
    double *gr = const_cast<double *>(T.gr), *gt = const_cast<double *>(T.gt), *gp = const_cast<double *>(T.gp);
    float *idr = const_cast<float *>(T.idr), *idt = const_cast<float *>(T.idt), *idp = const_cast<float *>(T.idp);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) gr[i] = rg[i];
    for (int i = threadIdx.x; i < nt; i += blockDim.x) gt[i] = tg[i];
    for (int i = threadIdx.x; i < np; i += blockDim.x) gp[i] = pg[i];
    for (int i = threadIdx.x; i < nr; i += blockDim.x) idr[i] = i + 1 < nr ? (float)(1.0 / (rg[i + 1] - rg[i])) : 0.0f;
    for (int i = threadIdx.x; i < nt; i += blockDim.x) idt[i] = i + 1 < nt ? (float)(1.0 / (tg[i + 1] - tg[i])) : 0.0f;
    for (int i = threadIdx.x; i < np; i += blockDim.x)
        idp[i] = (float)(1.0 / ((i + 1 < np ? pg[i + 1] : pg[0] + kTwoPi) - pg[i]));
    float *grf = const_cast<float *>(T.grf), *gtf = const_cast<float *>(T.gtf), *gpf = const_cast<float *>(T.gpf);
    for (int i = threadIdx.x; i < nr; i += blockDim.x) grf[i] = (float)rg[i];
    for (int i = threadIdx.x; i < nt; i += blockDim.x) gtf[i] = (float)tg[i];
    for (int i = threadIdx.x; i < np; i += blockDim.x) gpf[i] = (float)pg[i];
    if (threadIdx.x < 3) {
        const double *g = threadIdx.x == 0 ? rg : (threadIdx.x == 1 ? tg : pg);
        int n = threadIdx.x == 0 ? nr : (threadIdx.x == 1 ? nt : np);
        int kind = kSearch;
        double off = 0.0, inv = 0.0;
        // uniform model: g[i] ~ g0 + i d
        double d = (g[n - 1] - g[0]) / (n - 1);
        double dev = 0.0;
        for (int i = 0; i < n; ++i) dev = fmax(dev, fabs(g[i] - (g[0] + i * d)));
        if (dev <= 0.25 * d) {
            kind = kUniform;
            inv = 1.0 / d;
            off = g[0] * inv;
        } else if (g[0] > 0.0) {
            double dl = log(g[n - 1] / g[0]) / (n - 1);
            double devl = 0.0;
            for (int i = 0; i < n; ++i) devl = fmax(devl, fabs(log(g[i] / g[0]) - i * dl));
            if (devl <= 0.25 * dl) {
                kind = kGeometric;
                inv = 1.0 / dl;
                off = log(g[0]) * inv;
            }
        }
        if (threadIdx.x == 0) { h->kind_r = kind; h->off_r = off; h->inv_r = inv; h->foff_r = (float)off; h->finv_r = (float)inv; }
        if (threadIdx.x == 1) { h->kind_t = kind; h->off_t = off; h->inv_t = inv; h->foff_t = (float)off; h->finv_t = (float)inv; }
        if (threadIdx.x == 2) { h->kind_p = kind; h->off_p = off; h->inv_p = inv; h->foff_p = (float)off; h->finv_p = (float)inv; }
    }
    if (threadIdx.x == 0) {
        h->nr = nr;
        h->nt = nt;
        h->np = np;
    }
}

template <typename In, typename Out>
__global__ void pack_kernel(const In *__restrict__ in, int64_t cells, Out *__restrict__ rec, uint32_t *nonfinite) {
    uint32_t bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cells; i += (int64_t)gridDim.x * blockDim.x) {
        Out v[12];
#pragma unroll
        for (int k = 0; k < 11; ++k) {
            In x = in[11 * i + k];
            bad += !isfinite((double)x);
            v[k] = (Out)x;
        }
        v[11] = (Out)0;
        if constexpr (sizeof(Out) == 4) {
            float4 *o = reinterpret_cast<float4 *>(rec) + 3 * i;
            o[0] = make_float4(v[0], v[1], v[2], v[3]);
            o[1] = make_float4(v[4], v[5], v[6], v[7]);
            o[2] = make_float4(v[8], v[9], v[10], v[11]);
        } else {
            double2 *o = reinterpret_cast<double2 *>(rec) + 6 * i;
#pragma unroll
            for (int k = 0; k < 6; ++k) o[k] = make_double2(v[2 * k], v[2 * k + 1]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad && nonfinite) atomicAdd(nonfinite, bad);
}

// Same cell location as the fused renderer (locate_linear / locate_phi).
__global__ void locate_kernel(const void *tables, int nr, int nt, int np, const double *__restrict__ pts, int64_t n,
                              int32_t *__restrict__ index, float *__restrict__ weights) {
    Tables T = tables_at(tables, nr, nt, np);
    const TableHeader h = *T.h;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double r = pts[3 * i], th = pts[3 * i + 1], ph = pts[3 * i + 2];
        int32_t ir = -1, it = -1, ip = -1, valid = 0;
        float wr = 0.f, wt = 0.f, wp = 0.f;
        if (!(r < T.gr[0] || r > T.gr[nr - 1]) && !(th < T.gt[0] || th > T.gt[nt - 1]) && !isnan(r) && !isnan(th) &&
            isfinite(ph)) {
            valid = 1;
            ir = locate_linear(T.gr, nr, r, h.kind_r, h.off_r, h.inv_r);
            it = locate_linear(T.gt, nt, th, h.kind_t, h.off_t, h.inv_t);
            double p = wrap_phi(ph, T.gp[0]);
            ip = locate_phi(T.gp, np, p, h.kind_p, h.off_p, h.inv_p);
            double pp = p >= T.gp[ip] ? p : p + kTwoPi;
            wr = (float)(r - T.gr[ir]) * T.idr[ir];
            wt = (float)(th - T.gt[it]) * T.idt[it];
            wp = (float)(pp - T.gp[ip]) * T.idp[ip];
        }
        index[4 * i] = ir;
        index[4 * i + 1] = it;
        index[4 * i + 2] = ip;
        index[4 * i + 3] = valid;
        weights[3 * i] = wr;
        weights[3 * i + 1] = wt;
        weights[3 * i + 2] = wp;
    }
}

// FP32 FMA throughput probe (the denominator of the FP32 roofline): 8
// independent FMA chains per thread, so issue rate, not latency, bounds it.
__global__ void __launch_bounds__(256) fp32_peak_kernel(float *out, int iters, float seed) {
    float a0 = seed + threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
    float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

// FP64 probes: FMA chains as above, or 8 chains of x <- exp(-x) (values stay
// in (0, 1], converging to the omega constant; no overflow, no denormals).
__global__ void __launch_bounds__(256) fp64_peak_kernel(double *out, int iters, int mode, double seed) {
    double a0 = seed + threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
    double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
    if (mode == 0) {
        const double m = 0.999999, c = 1e-9;
        for (int i = 0; i < iters; ++i) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
                a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
            }
        }
    } else {
        for (int i = 0; i < iters; ++i) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                a0 = exp(-a0); a1 = exp(-a1); a2 = exp(-a2); a3 = exp(-a3);
                a4 = exp(-a4); a5 = exp(-a5); a6 = exp(-a6); a7 = exp(-a7);
            }
        }
    }
    const double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

static inline unsigned grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)(sm_count_current_device() > 0 ? sm_count_current_device() : 148) * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

static int check_grid_sizes(int64_t nr, int64_t nt, int64_t np) {
    if (nr < 2) return fail(BHN_ERR_VALUE, "r grid must contain at least 2 values");
    if (nt < 2) return fail(BHN_ERR_VALUE, "theta grid must contain at least 2 values");
    if (np < 2) return fail(BHN_ERR_VALUE, "phi grid must contain at least 2 values");
    if (nr > (1 << 20) || nt > (1 << 20) || np > (1 << 20)) return fail(BHN_ERR_VALUE, "coefficient brick shape is too large");
    return BHN_OK;
}

}  // namespace bhn

using namespace bhn;

extern "C" {

const char *bhn_core_version(void) { return "0.9.0+b200.1"; }

const char *bhn_last_error(void) { return g_last_error.c_str(); }

int bhn_device_info(int32_t *sm_count, int32_t *cc_major, int32_t *cc_minor, int64_t *global_mem_bytes) {
    int dev = 0;
    BHN_CUDA_TRY(cudaGetDevice(&dev));
    cudaDeviceProp p;
    BHN_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    if (global_mem_bytes) *global_mem_bytes = (int64_t)p.totalGlobalMem;
    return BHN_OK;
}

int bhn_stokes_rk2_brick(const double *coeffs, int64_t cells, double ds_cm, const double *initial, int64_t initial_len,
                         double *out, void *stream) {
    if (!std::isfinite(ds_cm) || ds_cm < 0.0) return fail(BHN_ERR_VALUE, "ds_cm must be finite and non-negative");
    if (cells <= 0) return fail(BHN_ERR_VALUE, "coeffs must contain one or more flat 11-coefficient cells");
    if (initial_len != 4 && initial_len != 4 * cells)
        return fail(BHN_ERR_VALUE, "initial must contain either 4 values or 4 values per coefficient cell");
    stokes_rk2_brick_kernel<<<grid_for(cells, 256), 256, 0, as_stream(stream)>>>(coeffs, cells, ds_cm, initial,
                                                                                 initial_len == 4, out);
    BHN_LAUNCH_CHECK("stokes_rk2_brick_kernel");
    return BHN_OK;
}

int bhn_stokes_exact_brick(const double *coeffs, int64_t cells, double ds_cm, const double *initial,
                           int64_t initial_len, double *out, void *stream) {
    if (!std::isfinite(ds_cm) || ds_cm < 0.0) return fail(BHN_ERR_VALUE, "ds_cm must be finite and non-negative");
    if (cells <= 0) return fail(BHN_ERR_VALUE, "coeffs must contain one or more flat 11-coefficient cells");
    if (initial_len != 4 && initial_len != 4 * cells)
        return fail(BHN_ERR_VALUE, "initial must contain either 4 values or 4 values per coefficient cell");
    stokes_exact_brick_kernel<<<grid_for(cells, 128), 128, 0, as_stream(stream)>>>(coeffs, cells, ds_cm, initial,
                                                                                   initial_len == 4, out);
    BHN_LAUNCH_CHECK("stokes_exact_brick_kernel");
    return BHN_OK;
}

int bhn_sample_brick_trilinear(const double *coeffs, const double *r_grid, int64_t nr, const double *theta_grid,
                               int64_t nt, const double *phi_grid, int64_t np, const double *points, int64_t n_points,
                               double *out, void *stream) {
    int rc = check_grid_sizes(nr, nt, np);
    if (rc) return rc;
    if (n_points < 0) return fail(BHN_ERR_VALUE, "points must contain flat r, theta, phi triples");
    if (n_points == 0) return BHN_OK;
    sample_trilinear_kernel<<<grid_for(n_points, 128), 128, 0, as_stream(stream)>>>(
        coeffs, r_grid, (int)nr, theta_grid, (int)nt, phi_grid, (int)np, points, n_points, out);
    BHN_LAUNCH_CHECK("sample_trilinear_kernel");
    return BHN_OK;
}

int bhn_sample_and_step_stokes(const double *coeffs, const double *r_grid, int64_t nr, const double *theta_grid,
                               int64_t nt, const double *phi_grid, int64_t np, const double *points, int64_t n_points,
                               double ds_cm, const double *initial, int64_t initial_len, int32_t invalid_policy,
                               double *out, void *stream) {
    if (!std::isfinite(ds_cm) || ds_cm < 0.0) return fail(BHN_ERR_VALUE, "ds_cm must be finite and non-negative");
    int rc = check_grid_sizes(nr, nt, np);
    if (rc) return rc;
    if (invalid_policy < 0 || invalid_policy > 2)
        return fail(BHN_ERR_VALUE, "invalid_policy must be 'nan', 'initial', or 'zero'");
    if (n_points < 0) return fail(BHN_ERR_VALUE, "points must contain flat r, theta, phi triples");
    if (initial_len != 4 && initial_len != 4 * n_points)
        return fail(BHN_ERR_VALUE, "initial must contain either 4 values or 4 values per sample point");
    if (n_points == 0) return BHN_OK;
    sample_and_step_kernel<<<grid_for(n_points, 128), 128, 0, as_stream(stream)>>>(
        coeffs, r_grid, (int)nr, theta_grid, (int)nt, phi_grid, (int)np, points, n_points, ds_cm, initial,
        initial_len == 4, invalid_policy, out);
    BHN_LAUNCH_CHECK("sample_and_step_kernel");
    return BHN_OK;
}

namespace {
struct SortLayout {
    int64_t keys_in, keys_out, idx_in, idx_out, temp, temp_bytes, total;
};

int key_bits(uint32_t max_key) {
    int b = 1;
    while (b < 32 && (max_key >> b)) ++b;
    return b;
}

// Offsets of the key / index arrays and the radix sort's temporary storage in
// the caller's scratch (each 256-byte aligned).  total < 0: unsupported sizes.
SortLayout sort_layout(int64_t n, int64_t cells) {
    SortLayout L{};
    L.total = -1;
    if (n <= 0 || n > INT32_MAX || cells <= 0 || cells >= (int64_t)UINT32_MAX) return L;
    size_t temp = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, temp, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                        (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0,
                                        key_bits((uint32_t)cells)) != cudaSuccess)
        return L;
    auto up = [](int64_t x) { return (x + 255) & ~(int64_t)255; };
    const int64_t a = up(4 * n);
    L.keys_in = 0;
    L.keys_out = a;
    L.idx_in = 2 * a;
    L.idx_out = 3 * a;
    L.temp = 4 * a;
    L.temp_bytes = (int64_t)temp;
    L.total = 4 * a + up((int64_t)temp);
    return L;
}
}  // namespace

int64_t bhn_sample_sort_scratch_bytes(int64_t n_points, int64_t cells) { return sort_layout(n_points, cells).total; }

namespace {
// The cell keys and their radix sort: idx_out (inside the scratch) receives the
// point indices in cell order.
int order_points_by_cell(const double *r_grid, int64_t nr, const double *theta_grid, int64_t nt, const double *phi_grid,
                         int64_t np, const double *points, int64_t n_points, const SortLayout &L, void *scratch,
                         void *stream, const uint32_t *&idx_out) {
    unsigned char *base = static_cast<unsigned char *>(scratch);
    uint32_t *keys_in = reinterpret_cast<uint32_t *>(base + L.keys_in);
    uint32_t *keys_out = reinterpret_cast<uint32_t *>(base + L.keys_out);
    uint32_t *idx_in = reinterpret_cast<uint32_t *>(base + L.idx_in);
    uint32_t *idx_sorted = reinterpret_cast<uint32_t *>(base + L.idx_out);
    const uint32_t cells = (uint32_t)(nr * nt * np);
    cudaStream_t s = as_stream(stream);
    cell_key_kernel<<<grid_for(n_points, 256), 256, 0, s>>>(r_grid, (int)nr, theta_grid, (int)nt, phi_grid, (int)np,
                                                          points, n_points, cells, keys_in, idx_in);
    BHN_LAUNCH_CHECK("cell_key_kernel");
    size_t temp = (size_t)L.temp_bytes;
    if (cub::DeviceRadixSort::SortPairs(base + L.temp, temp, keys_in, keys_out, idx_in, idx_sorted, (int)n_points, 0,
                                        key_bits(cells), s) != cudaSuccess)
        return fail(BHN_ERR_CUDA, "radix sort of the point cells failed");
    idx_out = idx_sorted;
    return BHN_OK;
}

int check_sort_scratch(int64_t n_points, int64_t cells, void *scratch, int64_t scratch_bytes, SortLayout &L) {
    L = sort_layout(n_points, cells);
    if (L.total < 0) return fail(BHN_ERR_VALUE, "point count or brick size outside the sorted path's range");
    if (!scratch || scratch_bytes < L.total || (reinterpret_cast<uintptr_t>(scratch) & 255))
        return fail(BHN_ERR_VALUE, "scratch must be 256-byte aligned and hold bhn_sample_sort_scratch_bytes bytes");
    return BHN_OK;
}
}  // namespace

int bhn_sample_brick_trilinear_sorted(const double *coeffs, const double *r_grid, int64_t nr, const double *theta_grid,
                                      int64_t nt, const double *phi_grid, int64_t np, const double *points,
                                      int64_t n_points, double *out, void *scratch, int64_t scratch_bytes,
                                      void *stream) {
    int rc = check_grid_sizes(nr, nt, np);
    if (rc) return rc;
    if (n_points < 0) return fail(BHN_ERR_VALUE, "points must contain flat r, theta, phi triples");
    if (n_points == 0) return BHN_OK;
    SortLayout L;
    rc = check_sort_scratch(n_points, nr * nt * np, scratch, scratch_bytes, L);
    if (rc) return rc;
    const uint32_t *order = nullptr;
    rc = order_points_by_cell(r_grid, nr, theta_grid, nt, phi_grid, np, points, n_points, L, scratch, stream, order);
    if (rc) return rc;
    sample_trilinear_ordered_kernel<<<grid_for(n_points, 128), 128, 0, as_stream(stream)>>>(
        coeffs, r_grid, (int)nr, theta_grid, (int)nt, phi_grid, (int)np, points, order, n_points, out);
    BHN_LAUNCH_CHECK("sample_trilinear_ordered_kernel");
    return BHN_OK;
}

int bhn_sample_and_step_stokes_sorted(const double *coeffs, const double *r_grid, int64_t nr,
                                      const double *theta_grid, int64_t nt, const double *phi_grid, int64_t np,
                                      const double *points, int64_t n_points, double ds_cm, const double *initial,
                                      int64_t initial_len, int32_t invalid_policy, double *out, void *scratch,
                                      int64_t scratch_bytes, void *stream) {
    if (!std::isfinite(ds_cm) || ds_cm < 0.0) return fail(BHN_ERR_VALUE, "ds_cm must be finite and non-negative");
    int rc = check_grid_sizes(nr, nt, np);
    if (rc) return rc;
    if (invalid_policy < 0 || invalid_policy > 2)
        return fail(BHN_ERR_VALUE, "invalid_policy must be 'nan', 'initial', or 'zero'");
    if (n_points < 0) return fail(BHN_ERR_VALUE, "points must contain flat r, theta, phi triples");
    if (initial_len != 4 && initial_len != 4 * n_points)
        return fail(BHN_ERR_VALUE, "initial must contain either 4 values or 4 values per sample point");
    if (n_points == 0) return BHN_OK;
    SortLayout L;
    rc = check_sort_scratch(n_points, nr * nt * np, scratch, scratch_bytes, L);
    if (rc) return rc;
    const uint32_t *idx_out = nullptr;
    rc = order_points_by_cell(r_grid, nr, theta_grid, nt, phi_grid, np, points, n_points, L, scratch, stream, idx_out);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    sample_and_step_ordered_kernel<<<grid_for(n_points, 128), 128, 0, s>>>(
        coeffs, r_grid, (int)nr, theta_grid, (int)nt, phi_grid, (int)np, points, idx_out, n_points, ds_cm, initial,
        initial_len == 4, invalid_policy, out);
    BHN_LAUNCH_CHECK("sample_and_step_ordered_kernel");
    return BHN_OK;
}

int bhn_sample_brick_valid_mask(const double *r_grid, int64_t nr, const double *theta_grid, int64_t nt,
                                const double *points, int64_t n_points, uint8_t *mask, void *stream) {
    if (nr < 2) return fail(BHN_ERR_VALUE, "r grid must contain at least 2 values");
    if (nt < 2) return fail(BHN_ERR_VALUE, "theta grid must contain at least 2 values");
    if (n_points <= 0) return n_points == 0 ? BHN_OK : fail(BHN_ERR_VALUE, "points must contain flat r, theta, phi triples");
    valid_mask_kernel<<<grid_for(n_points, 256), 256, 0, as_stream(stream)>>>(r_grid, (int)nr, theta_grid, (int)nt,
                                                                              points, n_points, mask);
    BHN_LAUNCH_CHECK("valid_mask_kernel");
    return BHN_OK;
}

int bhn_check_values(const double *values, int64_t n, int32_t check_increasing, uint32_t *counts, void *stream) {
    if (n <= 0) return BHN_OK;
    check_values_kernel<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(values, n, check_increasing, counts);
    BHN_LAUNCH_CHECK("check_values_kernel");
    return BHN_OK;
}

int bhn_fp32_peak_probe(float *scratch, int32_t iters, int32_t blocks_per_sm, int64_t *flops, void *stream) {
    const int sms = sm_count_current_device();
    if (sms <= 0) return fail(BHN_ERR_CUDA, "cannot query the SM count");
    if (iters < 1 || blocks_per_sm < 1 || blocks_per_sm > 32) return fail(BHN_ERR_VALUE, "bad probe size");
    const int threads = 256, blocks = sms * blocks_per_sm;
    fp32_peak_kernel<<<blocks, threads, 0, as_stream(stream)>>>(scratch, iters, 0.5f);
    BHN_LAUNCH_CHECK("fp32_peak_kernel");
    if (flops) *flops = (int64_t)blocks * threads * iters * 16 * 8 * 2;
    return BHN_OK;
}

int bhn_fp64_peak_probe(double *scratch, int32_t iters, int32_t blocks_per_sm, int32_t mode, int64_t *ops,
                        void *stream) {
    const int sms = sm_count_current_device();
    if (sms <= 0) return fail(BHN_ERR_CUDA, "cannot query the SM count");
    if (iters < 1 || blocks_per_sm < 1 || blocks_per_sm > 32) return fail(BHN_ERR_VALUE, "bad probe size");
    if (mode != 0 && mode != 1) return fail(BHN_ERR_VALUE, "probe mode must be 0 (fma) or 1 (exp)");
    const int threads = 256, blocks = sms * blocks_per_sm;
    fp64_peak_kernel<<<blocks, threads, 0, as_stream(stream)>>>(scratch, iters, mode, 0.5);
    BHN_LAUNCH_CHECK("fp64_peak_kernel");
    if (ops) *ops = (int64_t)blocks * threads * iters * (mode == 0 ? 16 * 8 * 2 : 4 * 8);
    return BHN_OK;
}

int64_t bhn_brick_tables_bytes(int32_t nr, int32_t nt, int32_t np) { return table_layout(nr, nt, np).total; }

int bhn_brick_build_tables(const double *r_grid, int32_t nr, const double *theta_grid, int32_t nt,
                           const double *phi_grid, int32_t np, void *tables, void *stream) {
    int rc = check_grid_sizes(nr, nt, np);
    if (rc) return rc;
    build_tables_kernel<<<1, 256, 0, as_stream(stream)>>>(r_grid, nr, theta_grid, nt, phi_grid, np, tables);
    BHN_LAUNCH_CHECK("build_tables_kernel");
    return BHN_OK;
}

int bhn_brick_pack(const void *coeffs, int32_t coeff_bytes, int64_t cells, void *records, int32_t record_bytes,
                   uint32_t *nonfinite, void *stream) {
    if (cells <= 0) return fail(BHN_ERR_VALUE, "coeffs must contain at least one cell");
    if ((coeff_bytes != 4 && coeff_bytes != 8) || (record_bytes != 4 && record_bytes != 8))
        return fail(BHN_ERR_VALUE, "brick values must be float32 or float64");
    if (reinterpret_cast<uintptr_t>(records) % 16 != 0) return fail(BHN_ERR_VALUE, "records must be 16-byte aligned");
    unsigned g = grid_for(cells, 256);
    cudaStream_t s = as_stream(stream);
    if (coeff_bytes == 4 && record_bytes == 4)
        pack_kernel<float, float><<<g, 256, 0, s>>>((const float *)coeffs, cells, (float *)records, nonfinite);
    else if (coeff_bytes == 8 && record_bytes == 4)
        pack_kernel<double, float><<<g, 256, 0, s>>>((const double *)coeffs, cells, (float *)records, nonfinite);
    else if (coeff_bytes == 4 && record_bytes == 8)
        pack_kernel<float, double><<<g, 256, 0, s>>>((const float *)coeffs, cells, (double *)records, nonfinite);
    else
        pack_kernel<double, double><<<g, 256, 0, s>>>((const double *)coeffs, cells, (double *)records, nonfinite);
    BHN_LAUNCH_CHECK("pack_kernel");
    return BHN_OK;
}

int bhn_brick_locate(const void *tables, int32_t nr, int32_t nt, int32_t np, const double *points, int64_t n_points,
                     int32_t *index, float *weights, void *stream) {
    int rc = check_grid_sizes(nr, nt, np);
    if (rc) return rc;
    if (n_points <= 0) return BHN_OK;
    locate_kernel<<<grid_for(n_points, 128), 128, 0, as_stream(stream)>>>(tables, nr, nt, np, points, n_points, index,
                                                                          weights);
    BHN_LAUNCH_CHECK("locate_kernel");
    return BHN_OK;
}

}  // extern "C"
