// bhn_internal.cuh -- shared definitions of the B200 GRRT hot-loop library.
//
// Reference citations are relative to the reference project root.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "blackhole_native.h"

namespace bhn {

// ---------------------------------------------------------------- host errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t err, const char *what);
int sm_count_current_device();

#define BHN_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return bhn::cuda_fail(e_, #expr); \
    } while (0)

#define BHN_LAUNCH_CHECK(what)                                   \
    do {                                                         \
        cudaError_t e_ = cudaGetLastError();                     \
        if (e_ != cudaSuccess) return bhn::cuda_fail(e_, what);  \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
constexpr double kEpsTheta = 1.0e-7;  // kerr.py:27

// ----------------------------------------------------------------- grid tables
// Grid kinds for the closed-form first guess of a cell index.  The guess is
// always followed by an exact fix-up against the stored knots, so the index
// equals numpy.searchsorted(side="right") - 1 for every grid; the kind only
// decides how many fix-up steps are needed.
enum GridKind : int32_t { kUniform = 0, kGeometric = 1, kSearch = 2 };

struct TableHeader {  // 128 bytes, at offset 0 of the tables buffer
    int32_t nr, nt, np, pad0;
    int32_t kind_r, kind_t, kind_p, pad1;
    // First guess f = X * inv - off with X = x (uniform) or X = log(x) (geometric).
    double off_r, inv_r, off_t, inv_t, off_p, inv_p;
    float foff_r, finv_r, foff_t, finv_t, foff_p, finv_p;  // the same in float
    double pad2[3];
};
static_assert(sizeof(TableHeader) == 128, "table header size");

// Offsets (bytes) inside the tables buffer: float64 knots, float32 reciprocal
// spacings, float32 knots (the FP32 kernel's copy).
struct TableLayout {
    int64_t gr, gt, gp, idr, idt, idp, grf, gtf, gpf, total;
};
__host__ __device__ inline TableLayout table_layout(int32_t nr, int32_t nt, int32_t np) {
    TableLayout L;
    L.gr = 128;
    L.gt = L.gr + 8 * (int64_t)nr;
    L.gp = L.gt + 8 * (int64_t)nt;
    L.idr = L.gp + 8 * (int64_t)np;
    L.idt = L.idr + 4 * (int64_t)nr;
    L.idp = L.idt + 4 * (int64_t)nt;
    L.grf = L.idp + 4 * (int64_t)np;
    L.gtf = L.grf + 4 * (int64_t)nr;
    L.gpf = L.gtf + 4 * (int64_t)nt;
    L.total = (L.gpf + 4 * (int64_t)np + 15) & ~(int64_t)15;
    return L;
}

struct Tables {
    const TableHeader *h;
    const double *gr, *gt, *gp;
    const float *idr, *idt, *idp;  // 1 / (g[i+1] - g[i]); idp[np-1] spans the wrap segment
    const float *grf, *gtf, *gpf;
};
__host__ __device__ inline Tables tables_at(const void *base, int32_t nr, int32_t nt, int32_t np) {
    TableLayout L = table_layout(nr, nt, np);
    const char *b = static_cast<const char *>(base);
    Tables t;
    t.h = reinterpret_cast<const TableHeader *>(b);
    t.gr = reinterpret_cast<const double *>(b + L.gr);
    t.gt = reinterpret_cast<const double *>(b + L.gt);
    t.gp = reinterpret_cast<const double *>(b + L.gp);
    t.idr = reinterpret_cast<const float *>(b + L.idr);
    t.idt = reinterpret_cast<const float *>(b + L.idt);
    t.idp = reinterpret_cast<const float *>(b + L.idp);
    t.grf = reinterpret_cast<const float *>(b + L.grf);
    t.gtf = reinterpret_cast<const float *>(b + L.gtf);
    t.gpf = reinterpret_cast<const float *>(b + L.gpf);
    return t;
}

// First index in [lo, hi) whose knot is > x (lib.rs:61-73 search_right).
template <typename T>
__device__ __forceinline__ int search_right(const T *g, int lo, int hi, T x) {
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (x < g[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Largest i in [0, n-2] with g[i] <= x, for g[0] <= x <= g[n-1]: the cell of
// native_kernels.py:137-146 (searchsorted right - 1, clamped; x == g[n-1]
// lands in cell n-2 with weight 1).
__device__ __forceinline__ int locate_linear(const double *g, int n, double x, int kind, double off, double inv) {
    int i;
    if (kind == kSearch) {
        i = search_right(g, 0, n, x) - 1;
    } else {
        float f = kind == kUniform ? (float)fma(x, inv, -off) : fmaf(__logf((float)x), (float)inv, -(float)off);
        i = (int)fmaxf(f, 0.0f);  // a guess only: clamped, then fixed up exactly
    }
    i = max(0, min(i, n - 2));
    while (i > 0 && x < g[i]) --i;
    while (i < n - 2 && x >= g[i + 1]) ++i;
    return i;
}

// Largest i in [0, n-1] with g[i] <= p for the wrapped phi p >= g[0]:
// native_kernels.py:149-161.
__device__ __forceinline__ int locate_phi(const double *g, int n, double p, int kind, double off, double inv) {
    int i;
    if (kind == kSearch) {
        i = search_right(g, 0, n, p) - 1;
    } else {
        i = (int)fmaxf((float)fma(p, inv, -off), 0.0f);
    }
    i = max(0, min(i, n - 1));
    while (i > 0 && p < g[i]) --i;
    while (i < n - 1 && p >= g[i + 1]) ++i;
    return i;
}

// The FP32 kernel's locators: the same searches over the float32 knots (exact
// for the float32 midpoints the FP32 kernel samples at).
// The closed-form guess of a uniform or geometric axis is within one cell of
// the answer: build_tables_kernel only classifies an axis so when every knot
// lies within a quarter cell of its model, which with FP32 rounding of the
// guess (~1e-4 cell) keeps floor(guess) in {i - 1, i, i + 1}; one step each
// way then gives searchsorted(side="right") - 1 exactly, without a loop.
__device__ __forceinline__ int locate_linear_f(const float *g, int n, float x, int kind, float off, float inv) {
    if (kind == kSearch) return max(0, min(search_right(g, 0, n, x) - 1, n - 2));
    const float f = kind == kUniform ? fmaf(x, inv, -off) : fmaf(__logf(x), inv, -off);
    int i = max(0, min((int)fmaxf(f, 0.0f), n - 2));
    i -= (i > 0 && x < g[i]) ? 1 : 0;
    i += (i < n - 2 && x >= g[i + 1]) ? 1 : 0;
    return i;
}

__device__ __forceinline__ int locate_phi_f(const float *g, int n, float p, int kind, float off, float inv) {
    if (kind == kSearch) return max(0, min(search_right(g, 0, n, p) - 1, n - 1));
    int i = max(0, min((int)fmaxf(fmaf(p, inv, -off), 0.0f), n - 1));
    i -= (i > 0 && p < g[i]) ? 1 : 0;
    i += (i < n - 1 && p >= g[i + 1]) ? 1 : 0;
    return i;
}

// native_kernels.py:133-134 / lib.rs:89-91: ((phi - base) mod 2 pi) + base.
__device__ __forceinline__ double wrap_phi(double phi, double base) {
    double m = fmod(phi - base, kTwoPi);
    if (m < 0.0) m += kTwoPi;
    return m + base;
}

// ------------------------------------------------------------- per-view table
struct __align__(16) ViewDev {
    double a, r_obs, theta_obs, phi_obs;
    double tan_y, tan_x, cos_roll, sin_roll;
    double pt_con, pphi_con0;          // p^t = 1/lapse, omega/lapse
    double e_r, e_th, e_ph;            // ZAMO tetrad scalings (kerr.py:144-148)
    double gcov00, gcov03, gcov11, gcov22, gcov33;
    double gcon00, gcon03, gcon11, gcon22, gcon33;
    double r_capture, escape_radius, r_plus, r_minus, r_photon;  // r_photon: innermost photon orbit
    double h_scale, h_min, h_max, L, max_tau;
    double width_d, height_d;          // image size as doubles (divisors of accelerated_renderer.py:138-140)
    int32_t width, height, x0, y0, crop_w, crop_h, max_steps, has_roll;
    int32_t valid, flags;
    int32_t axis_x0, axis_x1;          // crop-local columns [x0, x1) of the rays traced first (see setup_views_kernel)
    int64_t out_offset, ray_begin, ray_count, axis_begin;
};

struct QueueState {  // at offset 0 of the render scratch
    unsigned long long next;   // work-queue head (ray slots handed out)
    unsigned long long total;  // ray slots of all views
    uint32_t n_views, error_flags;
    uint32_t pad[10];
};
static_assert(sizeof(QueueState) == 64, "queue state size");

struct ScratchLayout {
    int64_t queue, stats, raw_views, views, ray_begin, axis_begin, total;
};
__host__ __device__ constexpr ScratchLayout scratch_layout(int32_t n_views) {
    ScratchLayout L{};
    L.queue = 0;
    L.stats = 64;
    L.raw_views = 256;
    L.views = (L.raw_views + (int64_t)sizeof(bhn_view) * n_views + 255) & ~(int64_t)255;
    L.ray_begin = (L.views + (int64_t)sizeof(ViewDev) * n_views + 255) & ~(int64_t)255;
    L.axis_begin = (L.ray_begin + 8 * ((int64_t)n_views + 1) + 255) & ~(int64_t)255;
    L.total = (L.axis_begin + 8 * ((int64_t)n_views + 1) + 255) & ~(int64_t)255;
    return L;
}

}  // namespace bhn
