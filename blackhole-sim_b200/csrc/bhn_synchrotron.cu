// bhn_synchrotron.cu -- coefficient-brick precompute on the GPU.
//
// The reference fills a brick cell by cell in Python
// (python/blackhole_sim/coefficient_bricks.py:119-152): per cell a local plasma
// frame (_fast_frame, :110-116) and the Hybrid synchrotron model
// (python/blackhole_sim/synchrotron.py:314-325), i.e. a thermal and a
// power-law component, each a pitch-angle-averaged (Gauss-Legendre) trapezoid
// integral over a Lorentz-factor grid of the F(x) / G(x) synchrotron kernels,
// looked up log-log in a 256-entry table (synchrotron.py:157-172).
//
// Here one warp owns a cell: its lanes split the Lorentz-factor nodes, each
// lane sums its nodes' contributions over all pitch nodes, and three warp
// reductions give the normalisation and the two integrals.  Everything is
// FP64.  Two rewrites that change rounding only:
//  * the trapezoid sum sum_i d_i (y_i + y_{i+1}) / 2 is evaluated as
//    sum_i c_i y_i with c_i = (d_{i-1} + d_i) / 2, which separates the
//    pitch sum from the Lorentz-factor sum;
//  * log x = log nu - log(1.5 nu_B sin a) - 2 log gamma instead of
//    log(nu / nu_c), so no logarithm is taken per (node, pitch) pair.
// The thermal distribution's normalisation theta_e K_2(1/theta_e)
// (synchrotron.py:189-196) cancels against its own trapezoid normalisation and
// is left out.  The kernel table's G(x) = x K_{2/3}(x) is computed on the host
// from the integral representation K_nu(x) = int_0^inf exp(-x cosh t)
// cosh(nu t) dt (DLMF 10.32.9) by the trapezoid rule.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "blackhole_native.h"
#include "bhn_internal.cuh"

namespace bhn {
namespace {

// python/blackhole_sim/calibration.py:18-25, synchrotron.py:177
constexpr double kC = 2.99792458e10;
constexpr double kMp = 1.67262192369e-24;
constexpr double kMe = 9.1093837015e-28;
constexpr double kKb = 1.380649e-16;
constexpr double kE = 4.80320471257e-10;
constexpr double kH = 6.62607015e-27;
constexpr double kPiD = 3.14159265358979323846;

constexpr int kTable = 256;      // synchrotron.py:158
constexpr int kMaxPitch = 64;
constexpr int kMaxGamma = 4096;

struct PitchSet {
    int n;
    double log_sin[kMaxPitch];   // log sin(alpha_m)
    double weight[kMaxPitch];    // 0.5 w_m sqrt(3) e^3 sin(alpha_m) / (m_e c^2): the pitch weight times pref / B
};

struct Component {
    int on, gamma_n;
    double p, gamma_min, gamma_max, fraction, absorption_scale, faraday_scale;  // power law
    double rotation_scale, conversion_scale;                                     // thermal
    PitchSet pitch;
};

struct SynchParams {
    double lx[kTable], lF[kTable], lG[kTable], sF[kTable], sG[kTable];  // log x knots, log F, log G, slopes
    double nu, log_nu, rho_unit, b_unit, mu_e_mp;
    Component th, nt;
    const double *rho, *theta_e, *b_con;
    void *out;
    int64_t cells;
    int out_bytes;
};

struct TableSmem {
    double lx[kTable], lF[kTable], lG[kTable], sF[kTable], sG[kTable];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// numpy.interp on the log-log table (synchrotron.py:165-172): knot j with
// lx[j] <= x < lx[j + 1]; x at or past the last knot takes the last value.
__device__ __forceinline__ void kernel_lookup(const TableSmem &T, double lx, double &F, double &G) {
    lx = fmin(fmax(lx, T.lx[0]), T.lx[kTable - 1]);
    if (lx >= T.lx[kTable - 1]) {
        F = exp(T.lF[kTable - 1]);
        G = exp(T.lG[kTable - 1]);
        return;
    }
    const double inv = (double)(kTable - 1) / (T.lx[kTable - 1] - T.lx[0]);
    int j = (int)((lx - T.lx[0]) * inv);
    j = max(0, min(j, kTable - 2));
    while (j > 0 && lx < T.lx[j]) --j;
    while (j < kTable - 2 && lx >= T.lx[j + 1]) ++j;
    const double d = __dsub_rn(lx, T.lx[j]);
    F = exp(__dadd_rn(__dmul_rn(T.sF[j], d), T.lF[j]));
    G = exp(__dadd_rn(__dmul_rn(T.sG[j], d), T.lG[j]));
}

// numpy.geomspace(start, stop, n)[i] (logspace of a linspace; exact end points).
__device__ __forceinline__ double geom_node(double start, double stop, double ls, double step, int i, int n) {
    if (i <= 0) return start;
    if (i >= n - 1) return stop;
    return pow(10.0, __dadd_rn(__dmul_rn((double)i, step), ls));
}

struct Integrals {
    double norm, I, Q;   // sum c_i f_i, sum c_i f_i sum_m W_m F, sum c_i f_i sum_m W_m G
};

// The pitch-averaged trapezoid integrals of synchrotron.py:207-237 for one
// distribution, split over the warp's lanes.  thermal: f = gamma^2 beta
// exp(-gamma / theta_e) on 1 + geomspace(1e-5, gmax - 1); power law: f =
// gamma^-p on geomspace(gamma_min, gamma_max).
__device__ Integrals integrate(const TableSmem &T, const Component &C, bool thermal, double theta_e, double base) {
    const int n = C.gamma_n, lane = threadIdx.x & 31;
    double g0, g1;
    if (thermal) {
        g0 = 1.0e-5;
        g1 = fmax(10.0, 1.0 + 45.0 * theta_e) - 1.0;
    } else {
        g0 = C.gamma_min;
        g1 = C.gamma_max;
    }
    const double ls = log10(g0), step = (log10(g1) - ls) / (double)(n - 1);
    const double inv_te = 1.0 / fmax(theta_e, 1.0e-12);
    Integrals acc = {0.0, 0.0, 0.0};
    for (int i = lane; i < n; i += 32) {
        const double xi = geom_node(g0, g1, ls, step, i, n);
        const double xm = i > 0 ? geom_node(g0, g1, ls, step, i - 1, n) : xi;
        const double xp = i < n - 1 ? geom_node(g0, g1, ls, step, i + 1, n) : xi;
        double gamma, c;
        if (thermal) {
            gamma = 1.0 + xi;
            c = 0.5 * ((i < n - 1 ? (1.0 + xp) - gamma : 0.0) + (i > 0 ? gamma - (1.0 + xm) : 0.0));
        } else {
            gamma = xi;
            c = 0.5 * ((xp - xi) + (xi - xm));
        }
        double f;
        if (thermal) {
            const double gm = fmax(gamma, 1.0);
            const double beta = sqrt(fmax(1.0 - 1.0 / (gm * gm), 0.0));
            f = gamma * gamma * beta * exp(-gamma * inv_te);
        } else {
            f = (gamma >= C.gamma_min && gamma <= C.gamma_max) ? pow(gamma, -C.p) : 0.0;
        }
        const double w = c * f;
        acc.norm += w;
        if (w != 0.0) {
            const double two_lg = 2.0 * log(gamma);
            double sI = 0.0, sQ = 0.0;
            for (int m = 0; m < C.pitch.n; ++m) {
                double F, G;
                kernel_lookup(T, base - C.pitch.log_sin[m] - two_lg, F, G);
                sI = fma(C.pitch.weight[m], F, sI);
                sQ = fma(C.pitch.weight[m], G, sQ);
            }
            acc.I += w * sI;
            acc.Q += w * sQ;
        }
    }
    acc.norm = warp_sum(acc.norm);
    acc.I = warp_sum(acc.I);
    acc.Q = warp_sum(acc.Q);
    return acc;
}

// synchrotron.py:175-182
__device__ __forceinline__ double planck_nu(double nu, double theta_e) {
    const double T = theta_e * kMe * kC * kC / kKb;
    const double x = kH * nu / fmax(kKb * T, 1.0e-300);
    if (x < 1.0e-3) return 2.0 * nu * nu * kKb * T / (kC * kC);
    return 2.0 * kH * nu * nu * nu / (kC * kC) / fmax(expm1(fmin(x, 700.0)), 1.0e-300);
}

// PolarizedCoefficients.rotated (synchrotron.py:67-77) of
// [jI, jQ, 0, 0, aI, aQ, 0, 0, rV, rQ, 0], added into out.
__device__ __forceinline__ void add_rotated(double *out, double jI, double jQ, double aI, double aQ, double rV,
                                            double rQ, double chi) {
    const double c = cos(2.0 * chi), s = sin(2.0 * chi);
    out[0] += jI;
    out[1] += jQ * c - 0.0 * s;
    out[2] += jQ * s + 0.0 * c;
    out[3] += 0.0;
    out[4] += aI;
    out[5] += aQ * c - 0.0 * s;
    out[6] += aQ * s + 0.0 * c;
    out[7] += 0.0;
    out[8] += rV;
    out[9] += rQ * c - 0.0 * s;
    out[10] += rQ * s + 0.0 * c;
}

__global__ void __launch_bounds__(128) precompute_kernel(const __grid_constant__ SynchParams P) {
    __shared__ TableSmem T;
    for (int i = threadIdx.x; i < kTable; i += blockDim.x) {
        T.lx[i] = P.lx[i];
        T.lF[i] = P.lF[i];
        T.lG[i] = P.lG[i];
        T.sF[i] = P.sF[i];
        T.sG[i] = P.sG[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t cell = warp; cell < P.cells; cell += warps) {
        // coefficient_bricks.py:110-116 with calibration.py:113-119
        const double b1 = P.b_con[4 * cell + 1], b2 = P.b_con[4 * cell + 2], b3 = P.b_con[4 * cell + 3];
        const double b_code = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(b1, b1), __dmul_rn(b2, b2)), __dmul_rn(b3, b3)));
        const double b = fmax(b_code * P.b_unit, 0.0);
        const double n_e = P.rho[cell] * P.rho_unit / P.mu_e_mp;
        const double chi = b_code > 0.0 ? atan2(b3, b2) : 0.0;  // atan2(b_vec[2], b_vec[1]) of b_vec = b_con[1:]
        const double te = fmax(P.theta_e[cell], 1.0e-8);
        double out[11];
#pragma unroll
        for (int k = 0; k < 11; ++k) out[k] = 0.0;
        if (n_e > 0.0 && b > 0.0 && P.nu > 0.0) {
            const double nu_B = kE * b / (2.0 * kPiD * kMe * kC);
            const double base = P.log_nu - log(1.5 * nu_B);
            const double b_par = b * 0.0;  // cos_pitch_to_los = 0 in the brick frame
            if (P.th.on) {  // synchrotron.py:248-275
                const Integrals r = integrate(T, P.th, true, te, base);
                const double inv = r.norm > 0.0 ? 1.0 / r.norm : 1.0;
                const double jI = n_e * (b * r.I * inv) / (4.0 * kPiD);
                const double jQ = n_e * (b * r.Q * inv) / (4.0 * kPiD);
                const double Bnu = planck_nu(P.nu, te);
                const double aI = jI / fmax(Bnu, 1.0e-300), aQ = jQ / fmax(Bnu, 1.0e-300);
                const double rel_supp = fmax(1.0 / (te * te + 1.0), 1.0e-8);
                double rV = P.th.rotation_scale * (kE * kE * kE / (kPiD * kMe * kMe * kC * kC));
                rV *= n_e * b_par / fmax(P.nu * P.nu, 1.0e-300) * rel_supp;
                double rQ = P.th.conversion_scale * (kE * kE * kE * kE / (4.0 * kPiD * kPiD * kMe * kMe * kMe * kC * kC * kC));
                rQ *= n_e * b * b / fmax(P.nu * P.nu * P.nu, 1.0e-300) * fmax(te, 1.0e-8);
                add_rotated(out, fmax(jI, 0.0), fmax(jQ, 0.0), fmax(aI, 0.0), fmax(aQ, 0.0), rV, rQ, chi);
            }
            if (P.nt.on && P.nt.fraction > 0.0) {  // synchrotron.py:290-311
                const Component &C = P.nt;
                const Integrals r = integrate(T, C, false, te, base);
                const double inv = 1.0 / fmax(r.norm, 1.0e-300);
                const double n_s = n_e * C.fraction;
                const double jI = n_s * (b * r.I * inv) / (4.0 * kPiD);
                double jQ = n_s * (b * r.Q * inv) / (4.0 * kPiD);
                const double cg = fmax(C.gamma_min, sqrt(fmax(P.nu / fmax(4.2e6 * b, 1.0e-300), 1.0)));
                const double energy = cg * kMe * kC * kC;
                const double aI = C.absorption_scale * jI / fmax(energy * P.nu * P.nu / (kC * kC), 1.0e-300);
                const double pol = fmin((C.p + 1.0) / (C.p + 7.0 / 3.0), 0.85);
                jQ = fmin(jQ, pol * jI);
                const double aQ = fmin(aI * pol, aI);
                double rV = C.faraday_scale * (kE * kE * kE / (kPiD * kMe * kMe * kC * kC));
                rV *= n_s * b_par / fmax(P.nu * P.nu, 1.0e-300) / fmax(C.gamma_min * C.gamma_min, 1.0);
                double rQ = C.faraday_scale * (kE * kE * kE * kE / (4.0 * kPiD * kPiD * kMe * kMe * kMe * kC * kC * kC));
                rQ *= n_s * b * b / fmax(P.nu * P.nu * P.nu, 1.0e-300) * log(fmax(C.gamma_max / C.gamma_min, 1.0));
                add_rotated(out, fmax(jI, 0.0), fmax(jQ, 0.0), fmax(aI, 0.0), fmax(aQ, 0.0), rV, rQ, chi);
            }
        }
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
    const double pref = std::sqrt(3.0) * kE * kE * kE / (kMe * kC * kC);  // synchrotron.py:185-186 per Gauss
    for (int m = 0; m < n; ++m) {
        const double sin_a = std::sqrt(std::max(0.0, 1.0 - x[m] * x[m]));
        if (!(sin_a > 0.0)) continue;  // Bp = B sin(alpha) <= 0 contributes nothing
        ps.log_sin[ps.n] = std::log(sin_a);
        ps.weight[ps.n] = 0.5 * w[m] * pref * sin_a;
        ++ps.n;
    }
}

}  // namespace
}  // namespace bhn

extern "C" int bhn_brick_precompute(const double *rho, const double *theta_e, const double *b_con, int64_t cells,
                                    const bhn_synchrotron_model *m, void *coeffs, int32_t coeff_bytes, void *stream) {
    using namespace bhn;
    if (!m) return fail(BHN_ERR_VALUE, "synchrotron model must not be NULL");
    if (cells < 1) return fail(BHN_ERR_VALUE, "the snapshot must contain at least one cell");
    if (!rho || !theta_e || !b_con || !coeffs) return fail(BHN_ERR_VALUE, "missing snapshot or output buffer");
    if (coeff_bytes != 4 && coeff_bytes != 8) return fail(BHN_ERR_VALUE, "brick values must be float32 or float64");
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
    static SynchParams P;  // ~10 KB: too large for the stack of some host threads; filled under the lock
    static std::mutex lock;
    std::lock_guard<std::mutex> g(lock);
    const HostTable &t = host_table();
    std::memcpy(P.lx, t.lx, sizeof t.lx);
    std::memcpy(P.lF, t.lF, sizeof t.lF);
    std::memcpy(P.lG, t.lG, sizeof t.lG);
    std::memcpy(P.sF, t.sF, sizeof t.sF);
    std::memcpy(P.sG, t.sG, sizeof t.sG);
    P.nu = m->nu_hz;
    P.log_nu = m->nu_hz > 0.0 ? std::log(m->nu_hz) : 0.0;
    P.rho_unit = m->rho_cgs_per_code;
    P.b_unit = m->b_gauss_per_code;
    P.mu_e_mp = std::max(m->mean_molecular_weight_per_electron * kMp, 1.0e-300);
    std::memset(&P.th, 0, sizeof P.th);
    std::memset(&P.nt, 0, sizeof P.nt);
    P.th.on = m->thermal != 0;
    if (P.th.on) {
        P.th.gamma_n = m->thermal_gamma_n;
        P.th.rotation_scale = m->thermal_rotation_scale;
        P.th.conversion_scale = m->thermal_conversion_scale;
        pitch_set(m->thermal_pitch_n, P.th.pitch);
    }
    P.nt.on = m->nonthermal != 0;
    if (P.nt.on) {
        P.nt.gamma_n = m->nonthermal_gamma_n;
        P.nt.p = m->nonthermal_p;
        P.nt.gamma_min = m->nonthermal_gamma_min;
        P.nt.gamma_max = m->nonthermal_gamma_max;
        P.nt.fraction = m->nonthermal_fraction;
        P.nt.absorption_scale = m->nonthermal_absorption_scale;
        P.nt.faraday_scale = m->nonthermal_faraday_scale;
        pitch_set(m->nonthermal_pitch_n, P.nt.pitch);
    }
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
