// bhn_synchrotron.cuh -- synchrotron transfer coefficients on the GPU (FP64).
//
// The Hybrid / thermal / power-law models of python/blackhole_sim/
// synchrotron.py:240-325: each component a pitch-angle-averaged
// (Gauss-Legendre) trapezoid integral over a Lorentz-factor grid of the
// F(x) / G(x) synchrotron kernels, looked up log-log in a 256-entry table
// (synchrotron.py:157-172).  One warp evaluates one plasma frame: its lanes
// split the Lorentz-factor nodes, each lane sums its nodes over all pitch
// nodes, and three warp reductions give the normalisation and the j_I, j_Q
// integrals.  Rewrites that change rounding only:
//  * the trapezoid sum sum_i d_i (y_i + y_{i+1}) / 2 is evaluated as
//    sum_i c_i y_i with c_i = (d_{i-1} + d_i) / 2, which separates the
//    pitch sum from the Lorentz-factor sum;
//  * log x = log nu - log(1.5 nu_B sin a) - 2 log gamma instead of
//    log(nu / nu_c), so no logarithm is taken per (node, pitch) pair.
// The thermal distribution's normalisation theta_e K_2(1/theta_e)
// (synchrotron.py:189-196) cancels against its own trapezoid normalisation and
// is left out.  The table's G(x) = x K_{2/3}(x) is computed on the host from
// the integral representation K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt
// (DLMF 10.32.9) by the trapezoid rule.
#pragma once

#include "blackhole_native.h"
#include "bhn_internal.cuh"

namespace bhn {
namespace synch {


// python/blackhole_sim/calibration.py:18-25, synchrotron.py:177
constexpr double kC = 2.99792458e10;
constexpr double kMp = 1.67262192369e-24;
constexpr double kMe = 9.1093837015e-28;
constexpr double kKb = 1.380649e-16;
constexpr double kE = 4.80320471257e-10;
constexpr double kH = 6.62607015e-27;
constexpr double kPiD = 3.14159265358979323846;

constexpr int kTable = 256;      // synchrotron.py:158
constexpr double kTailValue = 1.0e-250;  // F, G below this are dropped with their node (integrate)
constexpr int kMaxPitch = 64;
constexpr int kMaxGamma = 4096;

struct PitchSet {
    int n;
    double log_sin_max;          // the largest log sin(alpha_m) (the pitch with the smallest x)
    double log_sin[kMaxPitch];   // log sin(alpha_m)
    double weight[kMaxPitch];    // 0.5 w_m sqrt(3) e^3 sin(alpha_m) / (m_e c^2): the pitch weight times pref / B
};

struct Component {
    int on, gamma_n;
    double p, gamma_min, gamma_max, fraction, absorption_scale, faraday_scale;  // power law
    double rotation_scale, conversion_scale;                                     // thermal
    PitchSet pitch;
};

// The model in device form: kernel table, the two components and the plasma
// scaling of calibration.py:113-119 (n_e = rho rho_unit / (mu_e m_p), B = |b| b_unit).
struct Model {
    double lx[kTable], lF[kTable], lG[kTable], sF[kTable], sG[kTable];  // log x knots, log F, log G, slopes
    double lx_tail;  // from this log x on, F and G are below kTailValue up to the table end (+inf: nowhere)
    double rho_unit, b_unit, mu_e_mp;
    Component th, nt;
};

constexpr int kNodeCache = 256;  // power-law nodes kept per block (the default grid has 224)

struct TableSmem {
    double lx[kTable], lF[kTable], lG[kTable], sF[kTable], sG[kTable];
    double inv;      // (kTable - 1) / (lx[last] - lx[0]): knots per unit of log x
    double lx_tail;  // Model::lx_tail
    // The power law's nodes do not depend on the cell: its trapezoid weights
    // times gamma^-p and 2 log gamma, computed once per block (when it has at
    // most kNodeCache nodes), exactly as integrate() would per evaluation.
    int nt_cached;
    double nt_w[kNodeCache], nt_lg[kNodeCache];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// numpy.interp on the log-log table (synchrotron.py:165-172): knot j with
// lx[j] <= x < lx[j + 1]; x at or past the last knot takes the last value,
// x below the first the first (d = 0 there).  Every lane takes exactly two
// exp calls whatever its x, so a warp never runs the two cases one after the
// other.  The knots are log-uniform (log of a geomspace) to within a few ulps,
// so the first guess (x - lx[0]) / spacing is the right segment or one of its
// two neighbours (it can be off only within ~1e-13 of a knot): one
// conditional step each way, as selects rather than loops, finds the segment
// numpy.interp uses (2 % faster than the search loops, identical results).
__device__ __forceinline__ void kernel_lookup(const TableSmem &T, double lx, double &F, double &G) {
    const double lo = T.lx[0], hi = T.lx[kTable - 1];
    const bool past = lx >= hi;
    lx = fmin(fmax(lx, lo), hi);
    int j = (int)((lx - lo) * T.inv);
    j = max(0, min(j, kTable - 2));
    j -= (j > 0 && lx < T.lx[j]) ? 1 : 0;
    j += (j < kTable - 2 && lx >= T.lx[j + 1]) ? 1 : 0;
    const double d = __dsub_rn(lx, T.lx[j]);
    const double aF = past ? T.lF[kTable - 1] : __dadd_rn(__dmul_rn(T.sF[j], d), T.lF[j]);
    const double aG = past ? T.lG[kTable - 1] : __dadd_rn(__dmul_rn(T.sG[j], d), T.lG[j]);
    F = exp(aF);
    G = exp(aG);
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

// One node's pitch sums: W_m F(x_m), W_m G(x_m) over the distinct pitch angles,
// x_m = nu / (1.5 nu_B sin(alpha_m) gamma^2) as log x = base - log sin - 2 log gamma.
// A node whose smallest x (the pitch with the largest sin) already lies in
// the table's far tail adds terms below kTailValue times the pitch weights
// (< 1e-270): nothing a cell that emits can resolve.  Skipping it leaves such
// cells unchanged to the last bit (one that does not emit at all gets 0
// instead of a sum of those terms).
__device__ __forceinline__ void pitch_sums(const TableSmem &T, const PitchSet &ps, double base, double two_lg,
                                           double w, Integrals &acc) {
    if (!(w != 0.0 && __dsub_rn(__dsub_rn(base, ps.log_sin_max), two_lg) < T.lx_tail)) return;
    double sI = 0.0, sQ = 0.0;
    for (int m = 0; m < ps.n; ++m) {
        double F, G;
        kernel_lookup(T, base - ps.log_sin[m] - two_lg, F, G);
        sI = fma(ps.weight[m], F, sI);
        sQ = fma(ps.weight[m], G, sQ);
    }
    acc.I += w * sI;
    acc.Q += w * sQ;
}

// The pitch-averaged trapezoid integrals of synchrotron.py:207-237 for one
// distribution, split over the warp's lanes.  thermal: f = gamma^2 beta
// exp(-gamma / theta_e) on 1 + geomspace(1e-5, gmax - 1); power law: f =
// gamma^-p on geomspace(gamma_min, gamma_max).
static __device__ __noinline__ Integrals integrate(const TableSmem &T, const Component &C, bool thermal, double theta_e, double base) {
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
    if (!thermal && T.nt_cached) {
        for (int i = lane; i < n; i += 32) {
            const double w = T.nt_w[i];
            acc.norm += w;
            pitch_sums(T, C.pitch, base, T.nt_lg[i], w, acc);
        }
        acc.norm = warp_sum(acc.norm);
        acc.I = warp_sum(acc.I);
        acc.Q = warp_sum(acc.Q);
        return acc;
    }
    // Each lane evaluates one node per chunk of 32 (the next chunk's one step
    // ahead); the trapezoid's neighbours come from the adjacent lanes.
    double x_cur = geom_node(g0, g1, ls, step, lane, n), x_last = 0.0;
    for (int base0 = 0; base0 < n; base0 += 32) {
        const int i = base0 + lane;
        const double x_next = geom_node(g0, g1, ls, step, i + 32, n);
        double xm = __shfl_up_sync(0xffffffffu, x_cur, 1);
        double xp = __shfl_down_sync(0xffffffffu, x_cur, 1);
        const double next0 = __shfl_sync(0xffffffffu, x_next, 0);
        if (lane == 0) xm = x_last;   // node base0 - 1 (previous chunk's lane 31)
        if (lane == 31) xp = next0;   // node base0 + 32
        x_last = __shfl_sync(0xffffffffu, x_cur, 31);
        const double xi = x_cur;
        x_cur = x_next;
        if (i >= n) continue;
        if (i == 0) xm = xi;
        if (i == n - 1) xp = xi;
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
        pitch_sums(T, C.pitch, base, w != 0.0 ? 2.0 * log(gamma) : 0.0, w, acc);
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


// Block-cooperative copy of the kernel table into shared memory.
__device__ __forceinline__ void load_table(TableSmem &T, const Model &M) {
    for (int i = threadIdx.x; i < kTable; i += blockDim.x) {
        T.lx[i] = M.lx[i];
        T.lF[i] = M.lF[i];
        T.lG[i] = M.lG[i];
        T.sF[i] = M.sF[i];
        T.sG[i] = M.sG[i];
    }
    if (threadIdx.x == 0) {
        T.inv = (double)(kTable - 1) / (M.lx[kTable - 1] - M.lx[0]);
        T.lx_tail = M.lx_tail;
    }
    // the power law's nodes (integrate()'s arithmetic for them, once)
    const Component &C = M.nt;
    const bool cache = C.on && C.gamma_n <= kNodeCache;
    if (threadIdx.x == 0) T.nt_cached = cache;
    if (!cache) return;
    const int n = C.gamma_n;
    const double g0 = C.gamma_min, g1 = C.gamma_max;
    const double ls = log10(g0), step = (log10(g1) - ls) / (double)(n - 1);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double xi = geom_node(g0, g1, ls, step, i, n);
        const double xm = i > 0 ? geom_node(g0, g1, ls, step, i - 1, n) : xi;
        const double xp = i < n - 1 ? geom_node(g0, g1, ls, step, i + 1, n) : xi;
        const double c = 0.5 * ((xp - xi) + (xi - xm));
        const double f = (xi >= C.gamma_min && xi <= C.gamma_max) ? pow(xi, -C.p) : 0.0;
        const double w = c * f;
        T.nt_w[i] = w;
        T.nt_lg[i] = w != 0.0 ? 2.0 * log(xi) : 0.0;
    }
}

// The 11 coefficients of the model (synchrotron.py:248-325) for one local
// plasma frame (synchrotron.py:28-44): n_e [cm^-3], Theta_e (already floored),
// B [G] >= 0, cos of the pitch to the line of sight, EVPA chi, at frequency
// nu.  Warp-collective: every lane calls it with the same arguments and every
// lane gets the result.
__device__ inline void coefficients(const TableSmem &T, const Model &M, double n_e, double te, double b, double cos_los,
                             double chi, double nu, double out[11]) {
#pragma unroll
    for (int k = 0; k < 11; ++k) out[k] = 0.0;
    if (!(n_e > 0.0 && b > 0.0 && nu > 0.0)) return;
    const double b_perp = fabs(b) * sqrt(fmax(0.0, 1.0 - cos_los * cos_los));  // synchrotron.py:37-39
    const double b_par = b * cos_los;                                            // synchrotron.py:41-43
    const double nu_B = kE * b / (2.0 * kPiD * kMe * kC);
    const double base = log(nu) - log(1.5 * nu_B);
    const double K3 = kE * kE * kE / (kPiD * kMe * kMe * kC * kC);
    const double K4 = kE * kE * kE * kE / (4.0 * kPiD * kPiD * kMe * kMe * kMe * kC * kC * kC);
    if (M.th.on) {  // synchrotron.py:248-275
        const Integrals r = integrate(T, M.th, true, te, base);
        const double inv = r.norm > 0.0 ? 1.0 / r.norm : 1.0;
        const double jI = n_e * (b * r.I * inv) / (4.0 * kPiD);
        const double jQ = n_e * (b * r.Q * inv) / (4.0 * kPiD);
        const double Bnu = planck_nu(nu, te);
        const double aI = jI / fmax(Bnu, 1.0e-300), aQ = jQ / fmax(Bnu, 1.0e-300);
        const double rel_supp = fmax(1.0 / (te * te + 1.0), 1.0e-8);
        const double rV = M.th.rotation_scale * K3 * (n_e * b_par / fmax(nu * nu, 1.0e-300) * rel_supp);
        const double rQ = M.th.conversion_scale * K4 *
                          (n_e * b_perp * b_perp / fmax(nu * nu * nu, 1.0e-300) * fmax(te, 1.0e-8));
        add_rotated(out, fmax(jI, 0.0), fmax(jQ, 0.0), fmax(aI, 0.0), fmax(aQ, 0.0), rV, rQ, chi);
    }
    if (M.nt.on && M.nt.fraction > 0.0) {  // synchrotron.py:290-311
        const Component &C = M.nt;
        const Integrals r = integrate(T, C, false, te, base);
        const double inv = 1.0 / fmax(r.norm, 1.0e-300);
        const double n_s = n_e * C.fraction;
        const double jI = n_s * (b * r.I * inv) / (4.0 * kPiD);
        double jQ = n_s * (b * r.Q * inv) / (4.0 * kPiD);
        const double cg = fmax(C.gamma_min, sqrt(fmax(nu / fmax(4.2e6 * b_perp, 1.0e-300), 1.0)));
        const double energy = cg * kMe * kC * kC;
        const double aI = C.absorption_scale * jI / fmax(energy * nu * nu / (kC * kC), 1.0e-300);
        const double pol = fmin((C.p + 1.0) / (C.p + 7.0 / 3.0), 0.85);
        jQ = fmin(jQ, pol * jI);
        const double aQ = fmin(aI * pol, aI);
        const double rV = C.faraday_scale * K3 *
                          (n_s * b_par / fmax(nu * nu, 1.0e-300) / fmax(C.gamma_min * C.gamma_min, 1.0));
        const double rQ = C.faraday_scale * K4 *
                          (n_s * b_perp * b_perp / fmax(nu * nu * nu, 1.0e-300) *
                           log(fmax(C.gamma_max / C.gamma_min, 1.0)));
        add_rotated(out, fmax(jI, 0.0), fmax(jQ, 0.0), fmax(aI, 0.0), fmax(aQ, 0.0), rV, rQ, chi);
    }
}

// Host: the device model for a C model (kernel table built once per process).
int fill_model(const bhn_synchrotron_model *m, Model &out);

}  // namespace synch
}  // namespace bhn
