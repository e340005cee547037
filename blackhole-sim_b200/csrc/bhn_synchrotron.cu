// bhn_synchrotron.cu -- coefficient-brick precompute on the GPU.
//
// The reference fills a brick cell by cell in Python
// (python/blackhole_sim/coefficient_bricks.py:119-152): per cell a local plasma
// frame (_fast_frame, :110-116: no line-of-sight pitch) and the Hybrid
// synchrotron model (bhn_synchrotron.cuh).  Here one warp owns a cell.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "blackhole_native.h"
#include "bhn_internal.cuh"
#include "bhn_synchrotron.cuh"

namespace bhn {
namespace synch {

struct PrecomputeParams {
    Model M;
    double nu;
    const double *rho, *theta_e, *b_con;
    void *out;
    int64_t cells;
    int out_bytes;
};

__global__ void __launch_bounds__(128, 6) precompute_kernel(const __grid_constant__ PrecomputeParams P) {
    __shared__ TableSmem T;
    load_table(T, P.M);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t cell = warp; cell < P.cells; cell += warps) {
        // coefficient_bricks.py:110-116 with calibration.py:113-119
        const double b1 = P.b_con[4 * cell + 1], b2 = P.b_con[4 * cell + 2], b3 = P.b_con[4 * cell + 3];
        const double b_code = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(b1, b1), __dmul_rn(b2, b2)), __dmul_rn(b3, b3)));
        const double b = fmax(b_code * P.M.b_unit, 0.0);
        const double n_e = P.rho[cell] * P.M.rho_unit / P.M.mu_e_mp;
        const double chi = b_code > 0.0 ? atan2(b3, b2) : 0.0;  // atan2(b_vec[2], b_vec[1]) of b_vec = b_con[1:]
        const double te = fmax(P.theta_e[cell], 1.0e-8);
        double out[11];
        coefficients(T, P.M, n_e, te, b, 0.0, chi, P.nu, out);
        // the brick's dtype, then np.nan_to_num(nan=0, posinf=finfo.max, neginf=0) (coefficient_bricks.py:151)
        if (lane < 11) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 11; ++k) v = k == lane ? out[k] : v;
            if (P.out_bytes == 4) {
                float f = (float)v;
                f = isnan(f) ? 0.0f : (isinf(f) ? (f > 0.0f ? 3.402823466e38f : 0.0f) : f);
                reinterpret_cast<float *>(P.out)[11 * cell + lane] = f;
            } else {
                v = isnan(v) ? 0.0 : (isinf(v) ? (v > 0.0 ? 1.7976931348623157e308 : 0.0) : v);
                reinterpret_cast<double *>(P.out)[11 * cell + lane] = v;
            }
        }
    }
}

// The model's coefficients for given local plasma frames (synchrotron.py:248,
// :290, :318 -- ThermalSynchrotronCoefficients / NonthermalPowerLaw... /
// HybridSynchrotronCoefficients.coefficients(frame, nu_hz)): one warp per
// frame, frames[5 i .. 5 i + 4] = (n_e [cm^-3], Theta_e, B [G], cos of the pitch
// to the line of sight, EVPA), out[11 i .. 11 i + 10] in PolarizedCoefficients
// field order (the brick's COEFF_NAMES order).  Theta_e is taken as given: the
// reference's models floor it only where they divide by it.
struct FrameParams {
    Model M;
    double nu;
    const double *frames;
    double *out;
    int64_t n;
};

__global__ void __launch_bounds__(128, 6) frame_coefficients_kernel(const __grid_constant__ FrameParams P) {
    __shared__ TableSmem T;
    load_table(T, P.M);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < P.n; i += warps) {
        const double *f = P.frames + 5 * i;
        double out[11];
        coefficients(T, P.M, f[0], f[1], f[2], f[3], f[4], P.nu, out);
        if (lane < 11) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 11; ++k) v = k == lane ? out[k] : v;
            P.out[11 * i + lane] = v;
        }
    }
}

namespace {

// ------------------------------------------------------------ host tables
// K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt (DLMF 10.32.9), trapezoid
// rule with the step scaled to the integrand's width near t = 0 and the range
// cut where x (cosh t - 1) exceeds 750.
double bessel_k(double nu, double x) {
    const double h = std::min(0.02, 0.25 / std::sqrt(x));
    const double t_max = std::acosh(1.0 + 750.0 / x);
    double s = 0.5 * std::exp(-x);
    for (int k = 1;; ++k) {
        const double t = k * h;
        if (t > t_max + h) break;
        s += std::exp(-x * std::cosh(t)) * std::cosh(nu * t);
    }
    return h * s;
}

struct HostTable {
    double lx[kTable], lF[kTable], lG[kTable], sF[kTable], sG[kTable];
    double lx_tail;
};

// synchrotron.py:120-172: x = geomspace(1e-8, 1e3, 256), F(x) = 1.25 x^(1/3)
// exp(-x) (648 + x^2)^(1/12), G(x) = x K_{2/3}(x), stored as log values
// floored at log(1e-300), with numpy.interp's segment slopes.
const HostTable &host_table() {
    static HostTable t;
    static std::once_flag once;
    std::call_once(once, [] {
        const double ls = std::log10(1.0e-8), le = std::log10(1.0e3), step = (le - ls) / (kTable - 1);
        for (int i = 0; i < kTable; ++i) {
            double x = i == 0 ? 1.0e-8 : (i == kTable - 1 ? 1.0e3 : std::pow(10.0, (double)i * step + ls));
            const double xc = std::min(std::max(x, 1.0e-12), 1.0e3);
            double F = 1.25 * std::pow(xc, 1.0 / 3.0) * std::exp(-xc) * std::pow(648.0 + xc * xc, 1.0 / 12.0);
            double G = xc * bessel_k(2.0 / 3.0, xc);
            if (!std::isfinite(F)) F = 0.0;
            if (!std::isfinite(G)) G = 0.0;
            t.lx[i] = std::log(x);
            t.lF[i] = std::log(std::max(F, 1.0e-300));
            t.lG[i] = std::log(std::max(G, 1.0e-300));
        }
        for (int i = 0; i < kTable; ++i) {
            const int j = std::min(i, kTable - 2);
            t.sF[i] = (t.lF[j + 1] - t.lF[j]) / (t.lx[j + 1] - t.lx[j]);
            t.sG[i] = (t.lG[j + 1] - t.lG[j]) / (t.lx[j + 1] - t.lx[j]);
        }
        // first knot from which both log F and log G stay below log(kTailValue):
        // the linear segments in between stay below it too
        const double tail = std::log(kTailValue);
        int j0 = kTable;
        while (j0 > 0 && t.lF[j0 - 1] < tail && t.lG[j0 - 1] < tail) --j0;
        t.lx_tail = j0 < kTable ? t.lx[j0] : INFINITY;
    });
    return t;
}

// Gauss-Legendre nodes (ascending, as numpy.polynomial.legendre.leggauss) by
// Newton's method on P_n from the three-term recurrence.
void gauss_legendre(int n, double *x, double *w) {
    for (int k = 0; k < (n + 1) / 2; ++k) {
        double z = std::cos(kPiD * (k + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int l = 2; l <= n; ++l) {
                const double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) p0 = 1.0, p1 = z;
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int l = 2; l <= n; ++l) {
            const double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        const double wk = 2.0 / ((1.0 - z * z) * dp * dp);
        x[k] = -z;
        x[n - 1 - k] = z;
        w[k] = w[n - 1 - k] = wk;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

void pitch_set(int n, PitchSet &ps) {
    double x[kMaxPitch], w[kMaxPitch];
    gauss_legendre(n, x, w);
    ps.n = 0;
    ps.log_sin_max = 0.0;
    const double pref = std::sqrt(3.0) * kE * kE * kE / (kMe * kC * kC);  // synchrotron.py:185-186 per Gauss
    for (int m = 0; m < n; ++m) {
        const double sin_a = std::sqrt(std::max(0.0, 1.0 - x[m] * x[m]));
        if (!(sin_a > 0.0)) continue;  // Bp = B sin(alpha) <= 0 contributes nothing
        const double ls = std::log(sin_a), wt = 0.5 * w[m] * pref * sin_a;
        // the Gauss-Legendre nodes come in pairs +-mu with one sin(alpha) and one
        // weight: the pair's two lookups are the same numbers, so it is one node
        // of twice the weight
        int k = 0;
        while (k < ps.n && ps.log_sin[k] != ls) ++k;
        if (k < ps.n) {
            ps.weight[k] += wt;
            continue;
        }
        ps.log_sin[ps.n] = ls;
        ps.log_sin_max = ps.n == 0 ? ls : std::max(ps.log_sin_max, ls);
        ps.weight[ps.n] = wt;
        ++ps.n;
    }
}

}  // namespace

int fill_model(const bhn_synchrotron_model *m, Model &M) {
    if (!m) return fail(BHN_ERR_VALUE, "synchrotron model must not be NULL");
    if (!std::isfinite(m->nu_hz)) return fail(BHN_ERR_VALUE, "nu_hz must be finite");
    auto check_comp = [](int on, int gn, int pn) {
        return !on || (gn >= 2 && gn <= kMaxGamma && pn >= 1 && pn <= kMaxPitch);
    };
    if (!check_comp(m->thermal, m->thermal_gamma_n, m->thermal_pitch_n) ||
        !check_comp(m->nonthermal, m->nonthermal_gamma_n, m->nonthermal_pitch_n))
        return fail(BHN_ERR_VALUE, "gamma grids need 2.." + std::to_string(kMaxGamma) + " nodes and pitch averages 1.." +
                                       std::to_string(kMaxPitch) + " nodes");
    if (m->nonthermal && !(m->nonthermal_gamma_min > 0.0 && m->nonthermal_gamma_max > m->nonthermal_gamma_min))
        return fail(BHN_ERR_VALUE, "the power law needs 0 < gamma_min < gamma_max");
    const HostTable &t = host_table();
    std::memcpy(M.lx, t.lx, sizeof t.lx);
    std::memcpy(M.lF, t.lF, sizeof t.lF);
    std::memcpy(M.lG, t.lG, sizeof t.lG);
    std::memcpy(M.sF, t.sF, sizeof t.sF);
    std::memcpy(M.sG, t.sG, sizeof t.sG);
    M.lx_tail = t.lx_tail;
    M.rho_unit = m->rho_cgs_per_code;
    M.b_unit = m->b_gauss_per_code;
    M.mu_e_mp = std::max(m->mean_molecular_weight_per_electron * kMp, 1.0e-300);
    std::memset(&M.th, 0, sizeof M.th);
    std::memset(&M.nt, 0, sizeof M.nt);
    M.th.on = m->thermal != 0;
    if (M.th.on) {
        M.th.gamma_n = m->thermal_gamma_n;
        M.th.rotation_scale = m->thermal_rotation_scale;
        M.th.conversion_scale = m->thermal_conversion_scale;
        pitch_set(m->thermal_pitch_n, M.th.pitch);
    }
    M.nt.on = m->nonthermal != 0;
    if (M.nt.on) {
        M.nt.gamma_n = m->nonthermal_gamma_n;
        M.nt.p = m->nonthermal_p;
        M.nt.gamma_min = m->nonthermal_gamma_min;
        M.nt.gamma_max = m->nonthermal_gamma_max;
        M.nt.fraction = m->nonthermal_fraction;
        M.nt.absorption_scale = m->nonthermal_absorption_scale;
        M.nt.faraday_scale = m->nonthermal_faraday_scale;
        pitch_set(m->nonthermal_pitch_n, M.nt.pitch);
    }
    return BHN_OK;
}

}  // namespace synch
}  // namespace bhn

extern "C" int bhn_brick_precompute(const double *rho, const double *theta_e, const double *b_con, int64_t cells,
                                    const bhn_synchrotron_model *m, void *coeffs, int32_t coeff_bytes, void *stream) {
    using namespace bhn;
    using namespace bhn::synch;
    if (cells < 1) return fail(BHN_ERR_VALUE, "the snapshot must contain at least one cell");
    if (!rho || !theta_e || !b_con || !coeffs) return fail(BHN_ERR_VALUE, "missing snapshot or output buffer");
    if (coeff_bytes != 4 && coeff_bytes != 8) return fail(BHN_ERR_VALUE, "brick values must be float32 or float64");
    static PrecomputeParams P;  // ~10 KB: kept off the host stack; filled under the lock
    static std::mutex lock;
    std::lock_guard<std::mutex> g(lock);
    int rc = fill_model(m, P.M);
    if (rc) return rc;
    P.nu = m->nu_hz;
    P.rho = rho;
    P.theta_e = theta_e;
    P.b_con = b_con;
    P.out = coeffs;
    P.cells = cells;
    P.out_bytes = coeff_bytes;
    int dev = 0, sms = 148;
    BHN_CUDA_TRY(cudaGetDevice(&dev));
    BHN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t blocks = std::min<int64_t>((cells + 3) / 4, (int64_t)sms * 16);
    precompute_kernel<<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(P);
    BHN_LAUNCH_CHECK("precompute_kernel");
    return BHN_OK;
}

extern "C" int bhn_synchrotron_coefficients(const double *frames, int64_t n, const bhn_synchrotron_model *m,
                                            double *out, void *stream) {
    using namespace bhn;
    using namespace bhn::synch;
    if (n < 1) return fail(BHN_ERR_VALUE, "at least one plasma frame is required");
    if (!frames || !out) return fail(BHN_ERR_VALUE, "missing frame or output buffer");
    static FrameParams P;  // ~10 KB: kept off the host stack; filled under the lock
    static std::mutex lock;
    std::lock_guard<std::mutex> g(lock);
    int rc = fill_model(m, P.M);
    if (rc) return rc;
    P.nu = m->nu_hz;
    P.frames = frames;
    P.out = out;
    P.n = n;
    int dev = 0, sms = 148;
    BHN_CUDA_TRY(cudaGetDevice(&dev));
    BHN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t blocks = std::min<int64_t>((n + 3) / 4, (int64_t)sms * 16);
    frame_coefficients_kernel<<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(P);
    BHN_LAUNCH_CHECK("frame_coefficients_kernel");
    return BHN_OK;
}
