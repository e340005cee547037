// bhn_exact.cuh -- float64 helpers that reproduce the reference's arithmetic
// operation by operation (explicit round-to-nearest multiply / add / subtract,
// never contracted into FMAs): the Stokes RK2 step and the trilinear brick
// sampler with its bracket rules.  Shared by the micro-kernels and the
// physical (GRMHD snapshot) ray loop.
#pragma once

#include "bhn_internal.cuh"

namespace bhn {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// lib.rs:37-59 / native_kernels.py:213-222, evaluated left to right.
__device__ __forceinline__ void stokes_rhs_exact(const double s[4], const double c[11], double o[4]) {
    o[0] = sub(c[0], add(add(add(mul(c[4], s[0]), mul(c[5], s[1])), mul(c[6], s[2])), mul(c[7], s[3])));
    o[1] = sub(c[1], sub(add(add(mul(c[5], s[0]), mul(c[4], s[1])), mul(c[8], s[2])), mul(c[10], s[3])));
    o[2] = sub(c[2], add(add(sub(mul(c[6], s[0]), mul(c[8], s[1])), mul(c[4], s[2])), mul(c[9], s[3])));
    o[3] = sub(c[3], add(sub(add(mul(c[7], s[0]), mul(c[10], s[1])), mul(c[9], s[2])), mul(c[4], s[3])));
}

// lib.rs:210-225
__device__ __forceinline__ void stokes_step_rk2_exact(double s[4], const double c[11], double ds) {
    double k1[4], mid[4], k2[4];
    double hds = mul(0.5, ds);
    stokes_rhs_exact(s, c, k1);
    for (int i = 0; i < 4; ++i) mid[i] = add(s[i], mul(hds, k1[i]));
    stokes_rhs_exact(mid, c, k2);
    for (int i = 0; i < 4; ++i) s[i] = add(s[i], mul(ds, k2[i]));
}

// lib.rs:75-87 / native_kernels.py:137-146
__device__ __forceinline__ bool bracket_linear_exact(const double *g, int n, double x, int &i0, double &w) {
    if (x < g[0] || x > g[n - 1]) return false;
    if (x == g[n - 1]) {
        i0 = n - 2;
        w = 1.0;
        return true;
    }
    int lo = search_right(g, 0, n, x) - 1;
    lo = max(0, min(lo, n - 2));
    double den = sub(g[lo + 1], g[lo]);
    if (den < 1.0e-300) den = 1.0e-300;
    i0 = lo;
    w = sub(x, g[lo]) / den;
    return true;
}

// lib.rs:93-106 / native_kernels.py:149-161
__device__ __forceinline__ void bracket_phi_exact(const double *g, int n, double phi, int &i0, int &i1, double &w) {
    double p = wrap_phi(phi, g[0]);
    int lo = search_right(g, 0, n, p) - 1;
    if (lo < 0) lo = n - 1;
    if (lo >= n) lo = n - 1;
    int hi_i = (lo + 1) % n;
    double hi = hi_i > lo ? g[hi_i] : add(g[0], kTwoPi);
    double pp = p >= g[lo] ? p : add(p, kTwoPi);
    double den = sub(hi, g[lo]);
    if (den < 1.0e-300) den = 1.0e-300;
    i0 = lo;
    i1 = hi_i;
    w = sub(pp, g[lo]) / den;
}

// The trilinear blend of native_kernels.py:180-186: phi lerps, then theta, then r.
__device__ __forceinline__ bool lerp_cells(const double *__restrict__ coeffs, int nt, int np, int r0, int t0, int p0,
                                           int p1, double wr, double wt, double wp, double out[11]) {
    const int r1 = r0 + 1, t1 = t0 + 1;
    auto off = [&](int ir, int it, int ip) { return ((((int64_t)ir * nt + it) * np) + ip) * 11; };
    const double *c000 = coeffs + off(r0, t0, p0), *c001 = coeffs + off(r0, t0, p1);
    const double *c010 = coeffs + off(r0, t1, p0), *c011 = coeffs + off(r0, t1, p1);
    const double *c100 = coeffs + off(r1, t0, p0), *c101 = coeffs + off(r1, t0, p1);
    const double *c110 = coeffs + off(r1, t1, p0), *c111 = coeffs + off(r1, t1, p1);
    const double owp = sub(1.0, wp), owt = sub(1.0, wt), owr = sub(1.0, wr);
#pragma unroll
    for (int c = 0; c < 11; ++c) {
        double c00 = add(mul(owp, c000[c]), mul(wp, c001[c]));
        double c01 = add(mul(owp, c010[c]), mul(wp, c011[c]));
        double c10 = add(mul(owp, c100[c]), mul(wp, c101[c]));
        double c11 = add(mul(owp, c110[c]), mul(wp, c111[c]));
        double cc0 = add(mul(owt, c00), mul(wt, c01));
        double cc1 = add(mul(owt, c10), mul(wt, c11));
        out[c] = add(mul(owr, cc0), mul(wr, cc1));
    }
    return true;
}

// First-guess parameters of the three brick axes (r, theta, phi), classified
// once per block by its first warp: uniform when every knot lies within a
// quarter cell of g0 + k d, geometric when within a quarter cell of
// g0 exp(k dl), else binary search (the rule of build_tables_kernel).
struct AxisHints {
    int kind[3];
    double off[3], inv[3];
    double g0[3], gn[3];  // first and last knot
};

__device__ __forceinline__ void classify_axis_warp(const double *g, int n, int lane, int &kind, double &off,
                                                   double &inv) {
    kind = kSearch;
    off = inv = 0.0;
    const double d = (g[n - 1] - g[0]) / (n - 1);
    double dev = 0.0;
    for (int k = lane; k < n; k += 32) dev = fmax(dev, fabs(g[k] - (g[0] + k * d)));
    for (int o = 16; o > 0; o >>= 1) dev = fmax(dev, __shfl_xor_sync(0xffffffffu, dev, o));
    if (dev <= 0.25 * d) {
        kind = kUniform;
        inv = 1.0 / d;
        off = g[0] * inv;
        return;
    }
    if (!(g[0] > 0.0)) return;
    const double dl = log(g[n - 1] / g[0]) / (n - 1);
    double devl = 0.0;
    for (int k = lane; k < n; k += 32) devl = fmax(devl, fabs(log(g[k] / g[0]) - k * dl));
    for (int o = 16; o > 0; o >>= 1) devl = fmax(devl, __shfl_xor_sync(0xffffffffu, devl, o));
    if (devl <= 0.25 * dl) {
        kind = kGeometric;
        inv = 1.0 / dl;
        off = log(g[0]) * inv;
    }
}

// Every thread of the block must call this (it synchronises the block); the
// block needs at least one full warp.  NaN or unsorted knots classify as
// search, which is always exact.
__device__ __forceinline__ void load_axis_hints(AxisHints &h, const double *rg, int nr, const double *tg, int nt,
                                                const double *pg, int np) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        for (int a = 0; a < 3; ++a) {
            int kind;
            double off, inv;
            classify_axis_warp(a == 0 ? rg : (a == 1 ? tg : pg), a == 0 ? nr : (a == 1 ? nt : np), lane, kind, off,
                               inv);
            if (!(isfinite(off) && isfinite(inv))) kind = kSearch;
            if (lane == 0) {
                const double *g = a == 0 ? rg : (a == 1 ? tg : pg);
                const int n = a == 0 ? nr : (a == 1 ? nt : np);
                h.kind[a] = kind;
                h.off[a] = off;
                h.inv[a] = inv;
                h.g0[a] = g[0];
                h.gn[a] = g[n - 1];
            }
        }
    }
    __syncthreads();
}

// The cell of x (g0 <= x < gn) on an axis: largest i in [0, n-2] with
// g[i] <= x, as locate_linear, returned with g[i] and g[i+1].  On a classified
// axis (uniform or geometric: the closed-form guess is within one cell, see
// locate_linear_f) the guess's neighbours are loaded at once and the fix-up is
// a select; a guess found off by more (never on a classified axis) falls back
// to stepping.
__device__ __forceinline__ int locate_linear_sel(const double *g, int n, double x, int kind, double off, double inv,
                                                 double &gl, double &gh) {
    int i;
    if (kind == kSearch) {
        i = max(0, min(search_right(g, 0, n, x) - 1, n - 2));
    } else {
        const float f = kind == kUniform ? (float)fma(x, inv, -off) : fmaf(__logf((float)x), (float)inv, -(float)off);
        i = max(0, min((int)fmaxf(f, 0.0f), n - 2));
        const double gm = g[max(i - 1, 0)], gi = g[i], gi1 = g[i + 1], gp = g[min(i + 2, n - 1)];
        if (i > 0 && x < gi) {
            --i;
            gl = gm;
            gh = gi;
        } else if (i < n - 2 && x >= gi1) {
            ++i;
            gl = gi1;
            gh = gp;
        } else {
            gl = gi;
            gh = gi1;
        }
        if ((i == 0 || x >= gl) && (i == n - 2 || x < gh)) return i;
        while (i > 0 && x < g[i]) --i;
        while (i < n - 2 && x >= g[i + 1]) ++i;
    }
    gl = g[i];
    gh = g[i + 1];
    return i;
}

// The phi cell of the wrapped p >= g0: largest i in [0, n-1] with g[i] <= p,
// as locate_phi, returned with g[i] (the same select form).
__device__ __forceinline__ int locate_phi_sel(const double *g, int n, double p, int kind, double off, double inv,
                                              double &gl) {
    int i;
    if (kind == kSearch) {
        i = max(0, min(search_right(g, 0, n, p) - 1, n - 1));
    } else {
        i = max(0, min((int)fmaxf((float)fma(p, inv, -off), 0.0f), n - 1));
        const double gm = g[max(i - 1, 0)], gi = g[i], gi1 = g[min(i + 1, n - 1)], gp = g[min(i + 2, n - 1)];
        double gnext;
        if (i > 0 && p < gi) {
            --i;
            gl = gm;
            gnext = gi;
        } else if (i < n - 1 && p >= gi1) {
            ++i;
            gl = gi1;
            gnext = gp;
        } else {
            gl = gi;
            gnext = gi1;
        }
        if ((i == 0 || p >= gl) && (i == n - 1 || p < gnext)) return i;
        while (i > 0 && p < g[i]) --i;
        while (i < n - 1 && p >= g[i + 1]) ++i;
    }
    gl = g[i];
    return i;
}

// bracket_linear_exact with the cell found from the axis hint: the same cell
// (searchsorted(side="right") - 1) and the same weight for any sorted grid.
__device__ __forceinline__ bool bracket_linear_hinted(const double *g, int n, double x, int kind, double off,
                                                      double inv, double g0, double gn, int &i0, double &w) {
    if (x < g0 || x > gn) return false;
    if (x == gn) {
        i0 = n - 2;
        w = 1.0;
        return true;
    }
    double gl, gh;
    int lo;
    if (x == x) {
        lo = locate_linear_sel(g, n, x, kind, off, inv, gl, gh);
    } else {  // NaN: the search's answer
        lo = n - 2;
        gl = g[n - 2];
        gh = gn;
    }
    double den = sub(gh, gl);
    if (den < 1.0e-300) den = 1.0e-300;
    i0 = lo;
    w = sub(x, gl) / den;
    return true;
}

// bracket_phi_exact with the hinted cell search.
__device__ __forceinline__ void bracket_phi_hinted(const double *g, int n, double phi, int kind, double off,
                                                   double inv, double g0, int &i0, int &i1, double &w) {
    double p = wrap_phi(phi, g0);
    double gl;
    int lo;
    if (p >= g0) {
        lo = locate_phi_sel(g, n, p, kind, off, inv, gl);
    } else {  // below g0 or NaN: the search's answer
        lo = n - 1;
        gl = g[n - 1];
    }
    int hi_i = (lo + 1) % n;
    double hi = hi_i > lo ? g[hi_i] : add(g0, kTwoPi);
    double pp = p >= gl ? p : add(p, kTwoPi);
    double den = sub(hi, gl);
    if (den < 1.0e-300) den = 1.0e-300;
    i0 = lo;
    i1 = hi_i;
    w = sub(pp, gl) / den;
}

// lib.rs:171-208 / native_kernels.py:164-186
__device__ __forceinline__ bool sample_one_exact(const double *__restrict__ coeffs, const double *rg, int nr,
                                                 const double *tg, int nt, const double *pg, int np, double r,
                                                 double th, double ph, double out[11]) {
    int r0, t0, p0, p1;
    double wr, wt, wp;
    if (!bracket_linear_exact(rg, nr, r, r0, wr) || !bracket_linear_exact(tg, nt, th, t0, wt)) return false;
    bracket_phi_exact(pg, np, ph, p0, p1, wp);
    return lerp_cells(coeffs, nt, np, r0, t0, p0, p1, wr, wt, wp, out);
}

// sample_one_exact with the hinted brackets (same cells, weights and values).
__device__ __forceinline__ bool sample_one_hinted(const double *__restrict__ coeffs, const double *rg, int nr,
                                                  const double *tg, int nt, const double *pg, int np,
                                                  const AxisHints &h, double r, double th, double ph, double out[11]) {
    int r0, t0, p0, p1;
    double wr, wt, wp;
    if (!bracket_linear_hinted(rg, nr, r, h.kind[0], h.off[0], h.inv[0], h.g0[0], h.gn[0], r0, wr) ||
        !bracket_linear_hinted(tg, nt, th, h.kind[1], h.off[1], h.inv[1], h.g0[1], h.gn[1], t0, wt))
        return false;
    bracket_phi_hinted(pg, np, ph, h.kind[2], h.off[2], h.inv[2], h.g0[2], p0, p1, wp);
    return lerp_cells(coeffs, nt, np, r0, t0, p0, p1, wr, wt, wp, out);
}

// Cell records: the 11 channels of a cell and one pad, 16-byte aligned, in
// float32 (a float32 brick, 48 B, three 128-bit loads per cell) or float64
// (96 B, six).  A ray's eight corners sit at scattered addresses, so each warp
// load costs about one L1 wavefront per lane; 128-bit records cut the loads of
// a float32 brick's sample from 88 to 24.
template <typename T>
struct RecordVec;
template <>
struct RecordVec<float> {
    using V = float4;
    static constexpr int n = 4;
    __device__ static void widen(const float4 &v, double o[4]) {
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
};
template <>
struct RecordVec<double> {
    using V = double2;
    static constexpr int n = 2;
    __device__ static void widen(const double2 &v, double o[2]) {
        o[0] = v.x;
        o[1] = v.y;
    }
};

// The trilinear value of the 11 channels from the eight corner weights
// (products of the per-axis weights, formed once) and one fused multiply-add
// per corner and channel: 100 float64 operations instead of lerp_cells' 231
// separately rounded ones, equal to them within a few ulps.  Layout picks the
// corner loads: the [..][11] float64 brick (scalar loads) or 12-wide cell
// records in float32 / float64 (128-bit loads, values widened exactly).
template <typename T, int Stride>
__device__ __forceinline__ void lerp_weighted(const T *__restrict__ cells, int nt, int np, int r0, int t0, int p0,
                                              int p1, double wr, double wt, double wp, double out[11]) {
    const int r1 = r0 + 1, t1 = t0 + 1;
    auto cell = [&](int ir, int it, int ip) { return cells + ((((int64_t)ir * nt + it) * np) + ip) * Stride; };
    const T *q[8] = {cell(r0, t0, p0), cell(r0, t0, p1), cell(r0, t1, p0), cell(r0, t1, p1),
                     cell(r1, t0, p0), cell(r1, t0, p1), cell(r1, t1, p0), cell(r1, t1, p1)};
    const double owp = 1.0 - wp, owt = 1.0 - wt, owr = 1.0 - wr;
    const double a00 = owr * owt, a01 = owr * wt, a10 = wr * owt, a11 = wr * wt;
    const double w[8] = {a00 * owp, a00 * wp, a01 * owp, a01 * wp, a10 * owp, a10 * wp, a11 * owp, a11 * wp};
    if constexpr (Stride == 12) {
        using RV = RecordVec<T>;
        constexpr int W = RV::n;
#pragma unroll
        for (int g = 0; g < 12 / W; ++g) {
            double acc[W];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                double v[W];
                RV::widen(__ldg(reinterpret_cast<const typename RV::V *>(q[k]) + g), v);
#pragma unroll
                for (int j = 0; j < W; ++j) acc[j] = k == 0 ? w[0] * v[j] : fma(w[k], v[j], acc[j]);
            }
#pragma unroll
            for (int j = 0; j < W; ++j)
                if (g * W + j < 11) out[g * W + j] = acc[j];
        }
    } else {
#pragma unroll
        for (int c = 0; c < 11; ++c) {
            double acc = w[0] * __ldg(q[0] + c);
#pragma unroll
            for (int k = 1; k < 8; ++k) acc = fma(w[k], __ldg(q[k] + c), acc);
            out[c] = acc;
        }
    }
}

// sample_one_hinted's cells and per-axis weights, blended by lerp_weighted
// over the [..][Stride] cells (Stride 11: the reference's layout; 12: records).
template <typename T, int Stride>
__device__ __forceinline__ bool sample_weighted_hinted(const T *__restrict__ rec, const double *rg, int nr,
                                                      const double *tg, int nt, const double *pg, int np,
                                                      const AxisHints &h, double r, double th, double ph,
                                                      double out[11]) {
    int r0, t0, p0, p1;
    double wr, wt, wp;
    if (!bracket_linear_hinted(rg, nr, r, h.kind[0], h.off[0], h.inv[0], h.g0[0], h.gn[0], r0, wr) ||
        !bracket_linear_hinted(tg, nt, th, h.kind[1], h.off[1], h.inv[1], h.g0[1], h.gn[1], t0, wt))
        return false;
    bracket_phi_hinted(pg, np, ph, h.kind[2], h.off[2], h.inv[2], h.g0[2], p0, p1, wp);
    lerp_weighted<T, Stride>(rec, nt, np, r0, t0, p0, p1, wr, wt, wp, out);
    return true;
}

}  // namespace bhn
