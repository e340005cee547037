// bhn_learned.cuh -- learned step-size proposal for the fused ray kernel.
// Included at the end of bhn_render.cu (it shares its tracer pieces).
//
//   * adaptive_kernel: an RK2 step-doubling controller (FP32, compensated
//     positions).  Each attempt compares one step of h with two of h/2; the
//     Richardson estimate |y_{h/2,h/2} - y_h| / 3 in a mixed norm decides
//     acceptance, and h is rescaled by 0.9 err^(-1/3) (clamped).  Accepted
//     steps are recorded, with a hash-chosen probability, as training samples:
//     8 features of the state at the step start and log(h_opt / h_plain),
//     where h_opt = h err^(-1/3) is the step whose estimated RK2 error (O(h^3))
//     is exactly the tolerance and h_plain = clamp(h_scale r, h_min, h_max)
//     the plain step there.  h_opt is a function of the local state alone,
//     unlike the accepted h, which lags the controller's history; a network
//     fitted to the accepted h and fed its own previous proposal drifts.  The
//     kernel also renders the adaptive image with the brick accumulation of
//     accelerated_renderer.py:113-125.
//   * mlp_grad_kernel / mlp_adam_kernel / mlp_pack_kernel: training of the
//     8 -> 64 -> 64 -> 1 SiLU network (BF16 weights and activations, FP32
//     accumulation), forward and backward in FP32 SIMT with exactly the
//     roundings and activation of the inference path.
//   * learned_kernel: the ray loop with the network's proposal.  A warp
//     evaluates the network for its 32 rays with warp-level BF16
//     mma.sync.m16n8k16 (two m16 row tiles; each layer's accumulator tiles are
//     the next layer's A fragments), every `interval` steps.  The network
//     predicts log(h_opt / h_plain), the multiplier on the plain step at the
//     current r, floored at min_scale.  An embedded Euler-vs-midpoint
//     estimate h |k2 - k1| (O(h^2), two RHS evaluations like the plain step)
//     checks every proposal; where it fails (the network mispredicts, e.g.
//     rays grazing the spin axis) either the plain step (fallback 0) or the
//     step-doubling controller, started from 0.9 e^(-1/2) h (fallback 1),
//     takes that step, or (fallback 2) the step is not taken and that lane
//     tries it again next iteration with the proposal cut by 0.9 e^(-1/2), at
//     most max_attempts times.  With substeps = 2 a proposal is taken as two
//     RK2 steps of h / 2 under one brick segment, each half step checked.
//   * Both tracers cap steps inside the brick (brick_limit) and keep the
//     plain tracers' horizon guard (crosses_horizon).

namespace bhn {

// ------------------------------------------------------------ network blob
constexpr int kMlpParams = 8 * 64 + 64 + 64 * 64 + 64 + 64 + 1;  // W1 b1 W2 b2 W3 b3 (FP32 master)
constexpr int kOffW1 = 0, kOffB1 = 512, kOffW2 = 576, kOffB2 = 4672, kOffW3 = 4736, kOffB3 = 4800;

struct __align__(16) MlpNorm {
    float mu_x[8], inv_sx[8];  // feature standardisation
    float mu_y, sig_y;         // log h = mu_y + sig_y * y
    float pad[2];
};
static_assert(sizeof(MlpNorm) == 80, "norm size");

// Device blob read by the inference path: biases (FP32) and the BF16 weight
// fragments in mma.m16n8k16 B-operand order ([k tile][n tile][lane] -> 2 x b32).
struct __align__(16) MlpBlob {
    MlpNorm norm;
    float b1[64], b2[64], b3[4];
    uint2 w1f[8][32];      // K = 8 (padded to 16), N = 64
    uint2 w2f[4][8][32];   // K = 64, N = 64
    uint2 w3f[4][32];      // K = 64, N = 1 (padded to 8)
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// SiLU(z) = z * sigmoid(z) = z * (1 + tanh(z / 2)) / 2, with the hardware
// tanh approximation on a BF16 pair (the same instruction in training and
// inference, so both see the same activation).
__device__ __forceinline__ void tanh_bf16x2(float x0, float x1, float &t0, float &t1) {
    uint32_t in = pack_bf16x2(x0, x1), out;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(out) : "r"(in));
    const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(&out);
    t0 = __low2float(v);
    t1 = __high2float(v);
}
__device__ __forceinline__ void silu2(float z0, float z1, float &a0, float &a1, float &s0, float &s1) {
    float t0, t1;
    tanh_bf16x2(0.5f * z0, 0.5f * z1, t0, t1);
    s0 = fmaf(0.5f, t0, 0.5f);  // sigmoid
    s1 = fmaf(0.5f, t1, 0.5f);
    a0 = z0 * s0;
    a1 = z1 * s1;
}

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b.x), "r"(b.y));
}

// One network evaluation for the 32 rays of a warp (every lane calls it).
// f: this lane's 8 standardised features; xs: 128 b32 of per-warp shared
// scratch; ys: 32 floats of per-warp shared scratch.  Returns this lane's
// standardised output.
__device__ __forceinline__ float mlp_warp_infer(const float f[8], const MlpBlob &B, uint32_t *xs, float *ys) {
    const int lane = threadIdx.x & 31, gid = lane >> 2, t = lane & 3;
    reinterpret_cast<uint4 *>(xs)[lane] =
        make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]), pack_bf16x2(f[6], f[7]));
    __syncwarp();
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt) {
        const uint32_t x_lo = xs[(mt * 16 + gid) * 4 + t], x_hi = xs[(mt * 16 + gid + 8) * 4 + t];
        // layer 1: 16 x 16 (8 features + 8 zero columns) . 16 x 64
        float c1[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float bl = B.b1[nt * 8 + 2 * t], bh = B.b1[nt * 8 + 2 * t + 1];
            c1[nt][0] = bl; c1[nt][1] = bh; c1[nt][2] = bl; c1[nt][3] = bh;
            mma_bf16(c1[nt], x_lo, x_hi, 0u, 0u, B.w1f[nt][lane]);
        }
        uint32_t a2[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float p, q, r, s, u, v;
            silu2(c1[2 * j][0], c1[2 * j][1], p, q, u, v); a2[j][0] = pack_bf16x2(p, q);
            silu2(c1[2 * j][2], c1[2 * j][3], p, q, u, v); a2[j][1] = pack_bf16x2(p, q);
            silu2(c1[2 * j + 1][0], c1[2 * j + 1][1], p, q, u, v); a2[j][2] = pack_bf16x2(p, q);
            silu2(c1[2 * j + 1][2], c1[2 * j + 1][3], r, s, u, v); a2[j][3] = pack_bf16x2(r, s);
        }
        // layer 2: 16 x 64 . 64 x 64
        float c2[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float bl = B.b2[nt * 8 + 2 * t], bh = B.b2[nt * 8 + 2 * t + 1];
            c2[nt][0] = bl; c2[nt][1] = bh; c2[nt][2] = bl; c2[nt][3] = bh;
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) mma_bf16(c2[nt], a2[kt][0], a2[kt][1], a2[kt][2], a2[kt][3], B.w2f[kt][nt][lane]);
        }
        uint32_t a3[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float p, q, u, v;
            silu2(c2[2 * j][0], c2[2 * j][1], p, q, u, v); a3[j][0] = pack_bf16x2(p, q);
            silu2(c2[2 * j][2], c2[2 * j][3], p, q, u, v); a3[j][1] = pack_bf16x2(p, q);
            silu2(c2[2 * j + 1][0], c2[2 * j + 1][1], p, q, u, v); a3[j][2] = pack_bf16x2(p, q);
            silu2(c2[2 * j + 1][2], c2[2 * j + 1][3], p, q, u, v); a3[j][3] = pack_bf16x2(p, q);
        }
        // layer 3: 16 x 64 . 64 x 8 (column 0 is the output)
        float c3[4] = {t == 0 ? B.b3[0] : 0.0f, 0.0f, t == 0 ? B.b3[0] : 0.0f, 0.0f};
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) mma_bf16(c3, a3[kt][0], a3[kt][1], a3[kt][2], a3[kt][3], B.w3f[kt][lane]);
        if (t == 0) {
            ys[mt * 16 + gid] = c3[0];
            ys[mt * 16 + gid + 8] = c3[2];
        }
    }
    __syncwarp();
    const float y = ys[lane];
    __syncwarp();
    return y;
}

// FP32 parameters -> BF16 fragments (one block of 256 threads).
__global__ void mlp_pack_kernel(const float *__restrict__ P, MlpNorm norm, MlpBlob *__restrict__ blob) {
    const int tid = threadIdx.x;
    if (tid == 0) blob->norm = norm;
    for (int i = tid; i < 64; i += blockDim.x) {
        blob->b1[i] = P[kOffB1 + i];
        blob->b2[i] = P[kOffB2 + i];
    }
    if (tid < 4) blob->b3[tid] = tid == 0 ? P[kOffB3] : 0.0f;
    auto W = [&](int off, int kin, int nout, int k, int n) -> float {
        return (k < kin && n < nout) ? P[off + k * nout + n] : 0.0f;
    };
    for (int idx = tid; idx < 8 * 32; idx += blockDim.x) {  // layer 1
        const int nt = idx / 32, lane = idx % 32, gid = lane >> 2, t = lane & 3, n = nt * 8 + gid;
        blob->w1f[nt][lane] = make_uint2(pack_bf16x2(W(kOffW1, 8, 64, 2 * t, n), W(kOffW1, 8, 64, 2 * t + 1, n)),
                                         pack_bf16x2(W(kOffW1, 8, 64, 2 * t + 8, n), W(kOffW1, 8, 64, 2 * t + 9, n)));
    }
    for (int idx = tid; idx < 4 * 8 * 32; idx += blockDim.x) {  // layer 2
        const int kt = idx / 256, nt = (idx / 32) % 8, lane = idx % 32, gid = lane >> 2, t = lane & 3;
        const int n = nt * 8 + gid, k = kt * 16 + 2 * t;
        blob->w2f[kt][nt][lane] = make_uint2(pack_bf16x2(W(kOffW2, 64, 64, k, n), W(kOffW2, 64, 64, k + 1, n)),
                                             pack_bf16x2(W(kOffW2, 64, 64, k + 8, n), W(kOffW2, 64, 64, k + 9, n)));
    }
    for (int idx = tid; idx < 4 * 32; idx += blockDim.x) {  // layer 3
        const int kt = idx / 32, lane = idx % 32, gid = lane >> 2, t = lane & 3, k = kt * 16 + 2 * t;
        blob->w3f[kt][lane] = make_uint2(pack_bf16x2(W(kOffW3, 64, 1, k, gid), W(kOffW3, 64, 1, k + 1, gid)),
                                         pack_bf16x2(W(kOffW3, 64, 1, k + 8, gid), W(kOffW3, 64, 1, k + 9, gid)));
    }
}

// ------------------------------------------------------------ training
// One block = 128 samples.  Shared: BF16-rounded weights and biases, then the
// per-sample rows x, a1, a2, dz1, dz2, dy used by the block's weight-gradient
// reductions.  grad (FP32, kMlpParams) and loss are accumulated atomically.
constexpr int kTrainBlock = 128;
constexpr int kSampleStride = 9;  // 8 standardised features + standardised target

__host__ __device__ inline int64_t train_smem_bytes() {
    return 4 * ((int64_t)kMlpParams + 3 + (int64_t)kTrainBlock * (8 + 64 * 4 + 1));
}

__global__ void __launch_bounds__(kTrainBlock) mlp_grad_kernel(const float *__restrict__ P,
                                                                const float *__restrict__ samples,
                                                                const int64_t *__restrict__ index, int64_t first,
                                                                int64_t count, float *__restrict__ grad,
                                                                float *__restrict__ loss) {
    extern __shared__ __align__(16) float sm[];
    float *w = sm;                                   // kMlpParams (+3 pad)
    float *xs = w + kMlpParams + 3;                  // [128][8]
    float *a1s = xs + kTrainBlock * 8;               // [128][64]
    float *a2s = a1s + kTrainBlock * 64;             // [128][64]
    float *dz1s = a2s + kTrainBlock * 64;            // [128][64]
    float *dz2s = dz1s + kTrainBlock * 64;           // [128][64]
    float *dys = dz2s + kTrainBlock * 64;            // [128]
    const int tid = threadIdx.x;
    for (int i = tid; i < kMlpParams; i += blockDim.x) {
        const bool bias = (i >= kOffB1 && i < kOffW2) || (i >= kOffB2 && i < kOffW3) || i == kOffB3;
        w[i] = bias ? P[i] : bf16_round(P[i]);
    }
    __syncthreads();
    const int64_t s = (int64_t)blockIdx.x * kTrainBlock + tid;
    const bool live = s < count;
    const float *row = samples + (live ? index[first + s] : 0) * kSampleStride;
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = live ? bf16_round(row[k]) : 0.0f;
        xs[tid * 8 + k] = x[k];
    }
    const float target = live ? row[8] : 0.0f;
    // forward, layer 1 (z1 kept as sigmoid' in dz1s until the backward pass)
    for (int j = 0; j < 64; j += 2) {
        float z0 = w[kOffB1 + j], z1 = w[kOffB1 + j + 1];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            z0 = fmaf(x[k], w[kOffW1 + k * 64 + j], z0);
            z1 = fmaf(x[k], w[kOffW1 + k * 64 + j + 1], z1);
        }
        float a0, a1, s0, s1;
        silu2(z0, z1, a0, a1, s0, s1);
        a1s[tid * 64 + j] = bf16_round(a0);
        a1s[tid * 64 + j + 1] = bf16_round(a1);
        dz1s[tid * 64 + j] = fmaf(z0 * s0, 1.0f - s0, s0);  // SiLU'(z) = s + z s (1 - s)
        dz1s[tid * 64 + j + 1] = fmaf(z1 * s1, 1.0f - s1, s1);
    }
    // layer 2
    float y = w[kOffB3];
    for (int j = 0; j < 64; j += 2) {
        float z0 = w[kOffB2 + j], z1 = w[kOffB2 + j + 1];
        for (int i = 0; i < 64; ++i) {
            const float a = a1s[tid * 64 + i];
            z0 = fmaf(a, w[kOffW2 + i * 64 + j], z0);
            z1 = fmaf(a, w[kOffW2 + i * 64 + j + 1], z1);
        }
        float a0, a1, s0, s1;
        silu2(z0, z1, a0, a1, s0, s1);
        a0 = bf16_round(a0);
        a1 = bf16_round(a1);
        a2s[tid * 64 + j] = a0;
        a2s[tid * 64 + j + 1] = a1;
        dz2s[tid * 64 + j] = fmaf(z0 * s0, 1.0f - s0, s0);
        dz2s[tid * 64 + j + 1] = fmaf(z1 * s1, 1.0f - s1, s1);
        y = fmaf(a0, w[kOffW3 + j], y);
        y = fmaf(a1, w[kOffW3 + j + 1], y);
    }
    // backward: loss = mean (y - t)^2 over the batch
    const float err = live ? y - target : 0.0f;
    const float dy = 2.0f * err / (float)count;
    dys[tid] = dy;
    if (live) atomicAdd(loss, err * err);
    for (int j = 0; j < 64; ++j) dz2s[tid * 64 + j] *= dy * w[kOffW3 + j];
    for (int i = 0; i < 64; ++i) {
        float da = 0.0f;
        for (int j = 0; j < 64; ++j) da = fmaf(w[kOffW2 + i * 64 + j], dz2s[tid * 64 + j], da);
        dz1s[tid * 64 + i] *= da;
    }
    __syncthreads();
    // block reductions over the 128 samples
    for (int e = tid; e < 64 * 64; e += blockDim.x) {  // dW2
        const int i = e / 64, j = e % 64;
        float acc = 0.0f;
        for (int q = 0; q < kTrainBlock; ++q) acc = fmaf(a1s[q * 64 + i], dz2s[q * 64 + j], acc);
        atomicAdd(&grad[kOffW2 + e], acc);
    }
    for (int e = tid; e < 8 * 64; e += blockDim.x) {  // dW1
        const int k = e / 64, i = e % 64;
        float acc = 0.0f;
        for (int q = 0; q < kTrainBlock; ++q) acc = fmaf(xs[q * 8 + k], dz1s[q * 64 + i], acc);
        atomicAdd(&grad[kOffW1 + e], acc);
    }
    if (tid < 64) {
        float g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
        for (int q = 0; q < kTrainBlock; ++q) {
            g1 += dz1s[q * 64 + tid];
            g2 += dz2s[q * 64 + tid];
            g3 = fmaf(a2s[q * 64 + tid], dys[q], g3);
        }
        atomicAdd(&grad[kOffB1 + tid], g1);
        atomicAdd(&grad[kOffB2 + tid], g2);
        atomicAdd(&grad[kOffW3 + tid], g3);
    }
    if (tid == 64) {
        float g = 0.0f;
        for (int q = 0; q < kTrainBlock; ++q) g += dys[q];
        atomicAdd(&grad[kOffB3], g);
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; clears the gradient.
__global__ void mlp_adam_kernel(float *__restrict__ P, float *__restrict__ grad, float *__restrict__ m,
                                float *__restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float g = grad[i];
    const float mi = fmaf(b1, m[i], (1.0f - b1) * g);
    const float vi = fmaf(b2, v[i], (1.0f - b2) * g * g);
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    grad[i] = 0.0f;
}

// Network evaluation on given standardised feature rows (test hook for the
// inference path): out[i] = standardised output of row i.
__global__ void mlp_infer_kernel(const MlpBlob *__restrict__ blob, const float *__restrict__ feats, int64_t n,
                                 float *__restrict__ out) {
    __shared__ __align__(16) MlpBlob sb;
    __shared__ __align__(16) uint32_t xs[4][128];
    __shared__ float ys[4][32];
    for (int i = threadIdx.x; i < (int)(sizeof(MlpBlob) / 4); i += blockDim.x)
        reinterpret_cast<uint32_t *>(&sb)[i] = reinterpret_cast<const uint32_t *>(blob)[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    for (int64_t base = ((int64_t)blockIdx.x * 4 + warp) * 32; base < n; base += (int64_t)gridDim.x * 128) {
        const int64_t i = base + (threadIdx.x & 31);
        float f[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) f[k] = i < n ? feats[i * 8 + k] : 0.0f;
        const float y = mlp_warp_infer(f, sb, xs[warp], ys[warp]);
        if (i < n) out[i] = y;
    }
}

// ------------------------------------------------------------ adaptive and learned tracers
struct Geo {
    float rh, rl, th_h, th_l, ph_h, ph_l, pr, pth;
};

struct AdaptParams {
    float tol;          // step-doubling / embedded-check tolerance of the mixed norm
    float sample_prob;  // probability of recording an accepted step
    float h_floor, h_ceil;
    float margin;       // learned: log-h safety margin subtracted from the proposal
    float check_tol;    // learned: tolerance of the embedded check (0: no check)
    float brick_scale;  // in-brick step cap as a multiple of the plain step (0: none)
    float min_scale;    // learned: the step is at least min_scale times the plain step
    int interval;       // learned: steps between network evaluations
    int max_attempts;   // attempts per step before forcing acceptance (controller; learned retry)
    int fallback;       // learned: a failed check takes the plain step (0), the controller's (1), or retries (2)
    uint32_t seed;
    int substeps;       // learned: RK2 steps of h / substeps per brick segment (1 or 2)
};

// k1 at g and k2 at the Euler half step (the two stages of the RK2 midpoint step).
__device__ __forceinline__ void rk2_stages(const Geo &g, float h, const StepConst &C, float pt, float pphi, Deriv32 &k1,
                                           Deriv32 &k2, bool need_k1) {
    const float r0 = g.rh + g.rl;
    const bool south = g.th_h > kHalfPiF;
    const float d0 = south ? (kPiH - g.th_h) + (kPiL - g.th_l) : g.th_h + g.th_l;
    const float x0 = (g.rh - C.rp_h) + (g.rl - C.rp_l);
    float s, c;
    if (need_k1) {
        sincos_pole(d0, south, s, c);
        rhs32(r0, x0, s, c, g.pr, g.pth, pt, pphi, C.a, C.a2, C.dpm, k1);
    }
    const float hh = 0.5f * h;
    const float dm = fmaxf(south ? fmaf(-hh, k1.th, d0) : fmaf(hh, k1.th, d0), kEpsF);
    sincos_pole(dm, south, s, c);
    rhs32(fmaf(hh, k1.r, r0), fmaf(hh, k1.r, x0), s, c, fmaf(hh, k1.pr, g.pr), fmaf(hh, k1.pth, g.pth), pt, pphi,
          C.a, C.a2, C.dpm, k2);
}

__device__ __forceinline__ void rk2_k1(const Geo &g, const StepConst &C, float pt, float pphi, Deriv32 &k1) {
    const bool south = g.th_h > kHalfPiF;
    const float d0 = south ? (kPiH - g.th_h) + (kPiL - g.th_l) : g.th_h + g.th_l;
    float s, c;
    sincos_pole(d0, south, s, c);
    rhs32(g.rh + g.rl, (g.rh - C.rp_h) + (g.rl - C.rp_l), s, c, g.pr, g.pth, pt, pphi, C.a, C.a2, C.dpm, k1);
}

// Radiative-transfer limit of an error-controlled step.  The coefficient
// brick is sampled once per step at the step's midpoint (the plain method's
// rule), so its resolution is set by the step length, which the geodesic error
// norm does not see: inside the brick's (r, theta) box the step is capped at
// brick_scale times the plain step h = clamp(h_scale r, h_min, h_max); outside
// it, a step that would enter the box along k1 ends at most one such step
// past the entry point.  brick_scale <= 0 disables the limit.
__device__ __forceinline__ float brick_limit(float h, const Geo &g, const Deriv32 &k1, const StepConst &C,
                                             const Tables &T, int nr, int nt, float brick_scale) {
    if (!(brick_scale > 0.0f)) return h;
    const float r = g.rh + g.rl, th = g.th_h + g.th_l;
    const float r_in = T.grf[0], r_out = T.grf[nr - 1], t_lo = T.gtf[0], t_hi = T.gtf[nt - 1];
    const float hb = brick_scale * fminf(fmaxf(C.hs * fminf(r, r_out), C.hmin), C.hmax);
    const bool in_r = r >= r_in && r <= r_out, in_t = th >= t_lo && th <= t_hi;
    if (in_r && in_t) return fminf(h, hb);
    // affine time until each coordinate range is reached (0 when inside, inf when moving away)
    float tr = 0.0f, tt = 0.0f;
    if (!in_r) tr = r > r_out ? (k1.r < 0.0f ? (r - r_out) / -k1.r : INFINITY) : (k1.r > 0.0f ? (r_in - r) / k1.r : INFINITY);
    if (!in_t)
        tt = th < t_lo ? (k1.th > 0.0f ? (t_lo - th) / k1.th : INFINITY) : (k1.th < 0.0f ? (th - t_hi) / -k1.th : INFINITY);
    return fminf(h, fmaxf(tr, tt) + hb);
}

// The plain tracers' horizon guard: the trial step's midpoint (Euler half
// step) lies inside the horizon, so the step is not taken and the ray is
// captured.
__device__ __forceinline__ bool crosses_horizon(const Geo &g, const StepConst &C, float h, const Deriv32 &k1) {
    return fmaf(0.5f * h, k1.r, (g.rh - C.rp_h) + (g.rl - C.rp_l)) < 0.0f;
}

// g + h k2 with compensated positions, theta clamp and phi kept in [0, 2 pi).
__device__ __forceinline__ Geo geo_advance(const Geo &g, float h, const Deriv32 &k2) {
    Geo o = g;
    kahan_add(o.rh, o.rl, h * k2.r);
    kahan_add(o.th_h, o.th_l, h * k2.th);
    kahan_add(o.ph_h, o.ph_l, h * k2.ph);
    o.pr = fmaf(h, k2.pr, g.pr);
    o.pth = fmaf(h, k2.pth, g.pth);
    if (o.th_h + o.th_l < kEpsF) {
        o.th_h = kEpsF;
        o.th_l = 0.0f;
    } else if ((o.th_h - kTmaxH) + (o.th_l - kTmaxL) > 0.0f) {
        o.th_h = kTmaxH;
        o.th_l = kTmaxL;
    }
    if (o.ph_h >= kTwoPiH) {
        two_sum_add(o.ph_h, o.ph_l, -kTwoPiH);
        o.ph_l -= kTwoPiL;
    } else if (o.ph_h < 0.0f) {
        two_sum_add(o.ph_h, o.ph_l, kTwoPiH);
        o.ph_l += kTwoPiL;
    }
    return o;
}

// Mixed error norm: max over (r, theta, phi, p_r, p_theta) of |e_i| / (tol (1 + |y_i|)).
__device__ __forceinline__ float mixed_norm(float er, float eth, float eph, float epr, float epth, const Geo &g,
                                            float tol) {
    const float it = 1.0f / tol;
    float e = fabsf(er) / (1.0f + fabsf(g.rh));
    e = fmaxf(e, fabsf(eth) / (1.0f + fabsf(g.th_h)));
    e = fmaxf(e, fabsf(eph) / (1.0f + fabsf(g.ph_h)));
    e = fmaxf(e, fabsf(epr) / (1.0f + fabsf(g.pr)));
    e = fmaxf(e, fabsf(epth) / (1.0f + fabsf(g.pth)));
    return e * it;
}

// Step-doubling attempts from g (k1 = the derivatives at g) with trial step h:
// one step of h against two of h/2, Richardson estimate |y_{h/2,h/2} - y_h| / 3
// in units of the tolerance.  Returns the two-half-step solution of the
// accepted attempt; h is left at the accepted step and err at its estimate.
__device__ __forceinline__ Geo doubling_step(const Geo &g, float &h, Deriv32 &k1, const StepConst &C, float pt,
                                             float pphi, const AdaptParams &A, float &err,
                                             unsigned long long &n_eval, unsigned long long &n_rej) {
    Deriv32 k2;
    rk2_stages(g, h, C, pt, pphi, k1, k2, false);
    Geo y1 = geo_advance(g, h, k2), y2;
    for (int attempt = 0;; ++attempt) {
        Deriv32 k2h, k1b, k2b;
        rk2_stages(g, 0.5f * h, C, pt, pphi, k1, k2h, false);
        const Geo yh = geo_advance(g, 0.5f * h, k2h);
        rk2_stages(yh, 0.5f * h, C, pt, pphi, k1b, k2b, true);
        y2 = geo_advance(yh, 0.5f * h, k2b);
        n_eval += 5;
        err = mixed_norm((y2.rh - y1.rh) + (y2.rl - y1.rl), (y2.th_h - y1.th_h) + (y2.th_l - y1.th_l),
                         (y2.ph_h - y1.ph_h) + (y2.ph_l - y1.ph_l), y2.pr - y1.pr, y2.pth - y1.pth, g, A.tol) *
              (1.0f / 3.0f);
        if (!(err > 1.0f) || attempt + 1 >= A.max_attempts || h <= A.h_floor) break;
        ++n_rej;
        h = fmaxf(h * fmaxf(0.2f, 0.9f * __powf(err, -1.0f / 3.0f)), A.h_floor);
        rk2_stages(g, h, C, pt, pphi, k1, k2, false);
        y1 = geo_advance(g, h, k2);
    }
    return y2;
}

// Uniform [0, 1) from (ray, step, seed) by a 32-bit integer hash (splitmix-style mixing).
__device__ __forceinline__ float hash_uniform(uint32_t a, uint32_t b, uint32_t seed) {
    uint32_t x = a * 0x9E3779B9u ^ (b + 0x7F4A7C15u) * 0x85EBCA6Bu ^ seed * 0xC2B2AE35u;
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return (float)(x >> 8) * (1.0f / 16777216.0f);
}

// The brick segment of an accepted step (accelerated_renderer.py:113-125).
struct StokesAcc {
    float S0, S1, S2, S3, tau, jI;
    bool poison;
};
__device__ __forceinline__ bool brick_segment(const Tables &T, const float4 *__restrict__ rec, int nr, int nt, int np,
                                              const StepConst &C, const Geo &g0, const Geo &g1, float dr, float dph,
                                              StokesAcc &acc) {
    if (!(acc.tau < C.max_tau)) return false;
    const float r0 = g0.rh + g0.rl, th0 = g0.th_h + g0.th_l, ph0 = g0.ph_h + g0.ph_l, th1 = g1.th_h + g1.th_l;
    const float rmid = fmaf(0.5f, dr, r0), tmid = 0.5f * (th0 + th1), pmid = fmaf(0.5f, dph, ph0);
    if (rmid < T.grf[0] || rmid > T.grf[nr - 1] || tmid < T.gtf[0] || tmid > T.gtf[nt - 1]) return false;
    if (!(isfinite(rmid) && isfinite(tmid) && isfinite(pmid))) {
        acc.poison = true;
        return true;
    }
    const TableHeader &H = *T.h;
    const float gp0 = T.gpf[0];
    float pw = pmid - gp0;
    pw = fmaf(-kTwoPiH, floorf(pw * 0.159154943f), pw) + gp0;
    pw = fmaxf(pw, gp0);
    const int ir = locate_linear_f(T.grf, nr, rmid, H.kind_r, H.foff_r, H.finv_r);
    const int it = locate_linear_f(T.gtf, nt, tmid, H.kind_t, H.foff_t, H.finv_t);
    const int ip = locate_phi_f(T.gpf, np, pw, H.kind_p, H.foff_p, H.finv_p);
    const int ip1 = ip + 1 == np ? 0 : ip + 1;
    const float wr = (rmid - T.grf[ir]) * T.idr[ir], wt = (tmid - T.gtf[it]) * T.idt[it];
    const float wp = (pw - T.gpf[ip]) * T.idp[ip];
    const float owr = 1.0f - wr, owt = 1.0f - wt, owp = 1.0f - wp;
    const int64_t c00 = ((int64_t)ir * nt + it) * np;
    const int64_t cells[4] = {c00, c00 + np, c00 + (int64_t)nt * np, c00 + (int64_t)nt * np + np};
    const float wrt[4] = {owr * owt, owr * wt, wr * owt, wr * wt};
    float cf[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) cf[k] = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 *p0 = rec + 3 * (cells[q] + ip), *p1 = rec + 3 * (cells[q] + ip1);
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
    const float dth = th1 - th0;
    const float ds = C.L * fmaxf(sqrtf(fmaf(dr, dr, fmaf(dth, dth, dph * dph))), 1.0e-14f);
    const float j0 = cf[0], j1 = cf[1], j2 = cf[2], j3 = cf[3], ai = cf[4], aq = cf[5], au = cf[6], av = cf[7];
    const float rv = cf[8], rq = cf[9], ru = cf[10];
    float S0 = acc.S0, S1 = acc.S1, S2 = acc.S2, S3 = acc.S3;
    float k0 = j0 - (ai * S0 + aq * S1 + au * S2 + av * S3);
    float kq = j1 - (aq * S0 + ai * S1 + rv * S2 - ru * S3);
    float ku = j2 - (au * S0 - rv * S1 + ai * S2 + rq * S3);
    float kv = j3 - (av * S0 + ru * S1 - rq * S2 + ai * S3);
    const float hd = 0.5f * ds;
    const float m0 = fmaf(hd, k0, S0), m1 = fmaf(hd, kq, S1), m2 = fmaf(hd, ku, S2), m3 = fmaf(hd, kv, S3);
    k0 = j0 - (ai * m0 + aq * m1 + au * m2 + av * m3);
    kq = j1 - (aq * m0 + ai * m1 + rv * m2 - ru * m3);
    ku = j2 - (au * m0 - rv * m1 + ai * m2 + rq * m3);
    kv = j3 - (av * m0 + ru * m1 - rq * m2 + ai * m3);
    acc.S0 = fmaf(ds, k0, S0);
    acc.S1 = fmaf(ds, kq, S1);
    acc.S2 = fmaf(ds, ku, S2);
    acc.S3 = fmaf(ds, kv, S3);
    acc.tau = fmaf(fmaxf(ai, 0.0f), ds, acc.tau);
    acc.jI = j0;
    return true;
}

// The 8 network inputs at a state (before standardisation): log r, cos theta,
// p_r, p_theta, a, log|Delta|, p_phi (conserved along the ray), log of the
// last sampled j_I.
__device__ __forceinline__ void step_features(const Geo &g, const StepConst &C, float pphi, float jI, float f[8]) {
    const float r = g.rh + g.rl;
    const bool south = g.th_h > kHalfPiF;
    const float d0 = south ? (kPiH - g.th_h) + (kPiL - g.th_l) : g.th_h + g.th_l;
    float s, c;
    sincos_pole(d0, south, s, c);
    const float x = (g.rh - C.rp_h) + (g.rl - C.rp_l);
    f[0] = __logf(r);
    f[1] = c;
    f[2] = asinhf(g.pr);  // p_r grows like 1/Delta near the horizon
    f[3] = asinhf(g.pth);
    f[4] = C.a;
    f[5] = __logf(fabsf(x * (x + C.dpm)) + 1e-30f);
    f[6] = pphi;
    f[7] = __logf(fmaxf(jI, 0.0f) + 1e-12f);
}

// Termination after a step (kerr.py:364-377) on the compensated state.
__device__ __forceinline__ int terminate(const Geo &g, const StepConst &C, const StokesAcc &acc, float dr, bool finite,
                                         int steps) {
    if (!finite) return BHN_RAY_INVALID;
    if (acc.tau >= C.max_tau) return BHN_RAY_OPAQUE;
    if ((g.rh - C.rcap_h) + (g.rl - C.rcap_l) <= 0.0f) return BHN_RAY_CAPTURED;
    if (g.rh > C.esc && dr > 0.0f) return BHN_RAY_ESCAPED;
    if (steps >= C.max_steps) return BHN_RAY_MAX_STEPS;
    return -1;
}

__device__ __forceinline__ void write_stokes(void *out, uint32_t idx, const StokesAcc &a) {
    float4 o;
    o.x = (a.poison || !isfinite(a.S0)) ? 0.0f : a.S0;
    o.y = (a.poison || !isfinite(a.S1)) ? 0.0f : a.S1;
    o.z = (a.poison || !isfinite(a.S2)) ? 0.0f : a.S2;
    o.w = (a.poison || !isfinite(a.S3)) ? 0.0f : a.S3;
    reinterpret_cast<float4 *>(out)[idx] = o;
}

struct LearnParams {
    RenderParams R;
    AdaptParams A;
    float *samples;                      // adaptive: [capacity][9] raw (unstandardised) features + log h
    unsigned long long *sample_count;
    unsigned long long sample_capacity;
    const MlpBlob *blob;                 // learned
    unsigned long long *counters;        // [0] rk2 evaluations, [1] accepted steps, [2] rejected / fallbacks, [3] net evaluations
};

// Shared prologue of the adaptive and learned kernels: tables, view prefix and
// step constants in shared memory (the layout of the render kernel).
__device__ __forceinline__ void stage_shared(const RenderParams &P, unsigned char *smem, Tables &T, int64_t *&vbegin,
                                             StepConst *&sconst) {
    vbegin = reinterpret_cast<int64_t *>(smem + align16(P.tables_bytes));
    sconst = reinterpret_cast<StepConst *>(smem + align16(P.tables_bytes) + align16(8 * (P.n_views + 1)));
    const int4 *src = reinterpret_cast<const int4 *>(P.tables);
    int4 *dst = reinterpret_cast<int4 *>(smem);
    for (int i = threadIdx.x; i < P.tables_bytes / 16; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i <= P.n_views; i += blockDim.x) vbegin[i] = P.ray_begin[i];
    __syncthreads();
    T = tables_at(smem, P.nr, P.nt, P.np);
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
        c.r_guard = (float)fmin(v.r_photon, T.gr[0]);  // the adaptive and learned tracers always guard the horizon
        c.r_near = 0.0f;
        c.pad = 0.0f;
        c.max_steps = v.max_steps;
        c.pad1 = c.pad2 = c.pad3 = 0;
        sconst[i] = c;
    }
    __syncthreads();
}

__device__ __forceinline__ Geo camera_geo(const ViewDev &v, const CameraRay &c) {
    Geo g;
    split(v.r_obs, g.rh, g.rl);
    split(v.theta_obs, g.th_h, g.th_l);
    double p0 = fmod(v.phi_obs, kTwoPi);
    if (p0 < 0.0) p0 += kTwoPi;
    split(p0, g.ph_h, g.ph_l);
    g.pr = (float)c.pr;
    g.pth = (float)c.pth;
    return g;
}

// Step-doubling controller: renders the adaptive image and records samples.
// DRIFT: track each ray's Hamiltonian drift (only when it is asked for).
template <bool DRIFT>
__global__ void __launch_bounds__(256) adaptive_kernel(const LearnParams L) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RenderParams &P = L.R;
    Tables T;
    int64_t *vbegin;
    StepConst *sconst;
    stage_shared(P, smem, T, vbegin, sconst);
    const unsigned long long total = vbegin[P.n_views];
    const float4 *rec = reinterpret_cast<const float4 *>(P.records);
    const int lane = threadIdx.x & 31;
    unsigned long long n_eval = 0, n_acc = 0, n_rej = 0;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&P.q->next, 32ull);
        base = __shfl_sync(kFull, base, 0);
        if (base >= total) break;
        const unsigned long long slot = base + lane;
        if (slot < total) {
            const int vi = P.n_views == 1 ? 0 : find_view(vbegin, P.n_views, (int64_t)slot);
            const ViewDev &v = P.views[vi];
            const StepConst &C = sconst[vi];
            const PixelRef px = pixel_of(v, (int64_t)slot - vbegin[vi], P.tile_w, P.tile_h);
            const CameraRay cam = camera_ray(v, px.px, px.py);
            const float pt = (float)cam.pt, pphi = (float)cam.pphi;
            Geo g = camera_geo(v, cam);
            const float H0 = DRIFT ? (float)cam.H0 : 0.0f;
            float drift = 0.0f;  // max | |H| - |H0| | over the accepted steps' starts (kerr.py:352, 367)
            StokesAcc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, false};
            // first trial step 0.05 r: the controller then tracks the accepted step
            // without a long ramp from a small start (which would dominate the samples)
            float h = fminf(fmaxf(0.05f * (g.rh + g.rl), L.A.h_floor), L.A.h_ceil);
            int steps = 0, st = -1;
            while (st < 0) {
                if (g.rh < C.r_guard && g.pr < 0.0f) {
                    st = BHN_RAY_CAPTURED;
                    break;
                }
                Deriv32 k1;
                rk2_k1(g, C, pt, pphi, k1);
                if constexpr (DRIFT) drift = fmaxf(drift, fabsf(fabsf(k1.H) - H0));
                h = fmaxf(brick_limit(h, g, k1, C, T, P.nr, P.nt, L.A.brick_scale), L.A.h_floor);
                if (crosses_horizon(g, C, h, k1)) {
                    st = BHN_RAY_CAPTURED;
                    break;
                }
                float err = 0.0f;
                const Geo y2 = doubling_step(g, h, k1, C, pt, pphi, L.A, err, n_eval, n_rej);
                // record (features at the step start, log(h_opt / h_plain)); err is floored at
                // 1e-6 so a step held back by the growth cap extrapolates at most 100x
                if (L.samples && hash_uniform((uint32_t)slot, (uint32_t)steps, L.A.seed) < L.A.sample_prob) {
                    const unsigned long long k = atomicAdd(L.sample_count, 1ull);
                    if (k < L.sample_capacity) {
                        float f[8];
                        step_features(g, C, pphi, acc.jI, f);
                        float *o = L.samples + k * kSampleStride;
#pragma unroll
                        for (int q = 0; q < 8; ++q) o[q] = f[q];
                        const float h_opt = h * __powf(fmaxf(err, 1e-6f), -1.0f / 3.0f);
                        const float h_plain = fminf(fmaxf(C.hs * (g.rh + g.rl), C.hmin), C.hmax);
                        o[8] = __logf(fminf(fmaxf(h_opt, L.A.h_floor), L.A.h_ceil) / h_plain);
                    }
                }
                const float dr = (y2.rh - g.rh) + (y2.rl - g.rl), dph = (y2.ph_h - g.ph_h) + (y2.ph_l - g.ph_l);
                const float dph_u = dph > 3.14159f ? dph - kTwoPiH : (dph < -3.14159f ? dph + kTwoPiH : dph);
                brick_segment(T, rec, P.nr, P.nt, P.np, C, g, y2, dr, dph_u, acc);
                const bool finite = isfinite(y2.rh + y2.th_h + y2.ph_h + y2.pr + y2.pth);
                g = y2;
                ++steps;
                ++n_acc;
                h = fminf(fmaxf(h * fminf(2.0f, fmaxf(0.3f, 0.9f * __powf(fmaxf(err, 1e-6f), -1.0f / 3.0f))),
                                L.A.h_floor),
                          L.A.h_ceil);
                st = terminate(g, C, acc, dr, finite, steps);
            }
            write_stokes(P.out, (uint32_t)px.out_idx, acc);
            if (P.ray_steps) P.ray_steps[px.out_idx] = steps;
            if (P.ray_status) P.ray_status[px.out_idx] = (uint8_t)st;
            if constexpr (DRIFT) P.ray_drift[px.out_idx] = drift;
        }
        __syncwarp();
    }
    if (L.counters) {
        atomicAdd(&L.counters[0], n_eval);
        atomicAdd(&L.counters[1], n_acc);
        atomicAdd(&L.counters[2], n_rej);
    }
}

// The ray loop with the network's step proposal (FP32, horizon guard on).
// DRIFT: track each ray's Hamiltonian drift (only when it is asked for: the two
// registers it holds cost occupancy); SUBSTEPS: RK2 steps per brick segment.
// Five 128-thread blocks per SM: at most 102 registers a thread.
template <bool DRIFT, int SUBSTEPS>
__global__ void __launch_bounds__(128, 5) learned_kernel(const LearnParams L) {
    extern __shared__ __align__(16) unsigned char smem[];
    const RenderParams &P = L.R;
    Tables T;
    int64_t *vbegin;
    StepConst *sconst;
    stage_shared(P, smem, T, vbegin, sconst);
    __shared__ __align__(16) MlpBlob sb;
    __shared__ __align__(16) uint32_t xs_all[4][128];
    __shared__ float ys_all[4][32];
    for (int i = threadIdx.x; i < (int)(sizeof(MlpBlob) / 4); i += blockDim.x)
        reinterpret_cast<uint32_t *>(&sb)[i] = reinterpret_cast<const uint32_t *>(L.blob)[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *xs = xs_all[warp];
    float *ys = ys_all[warp];
    const unsigned long long total = vbegin[P.n_views];
    const float4 *rec = reinterpret_cast<const float4 *>(P.records);
    const MlpNorm &N = sb.norm;
    unsigned long long n_eval = 0, n_acc = 0, n_fb = 0, n_net = 0;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&P.q->next, 32ull);
        base = __shfl_sync(kFull, base, 0);
        if (base >= total) break;
        const unsigned long long slot = base + lane;
        bool alive = slot < total;
        int vi = 0;
        PixelRef px;
        px.px = px.py = 0;
        px.out_idx = 0;
        Geo g = {1000.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float pt = -1.0f, pphi = 0.0f, mult = 1.0f, H0 = 0.0f, drift = 0.0f;
        float shrink = 1.0f;  // retry fallback: this lane's cut of the proposal since the last evaluation
        int fails = 0;        // retry fallback: failed attempts at the current step
        StokesAcc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, false};
        int steps = 0, st = -1;
        if (alive) {
            vi = P.n_views == 1 ? 0 : find_view(vbegin, P.n_views, (int64_t)slot);
            const ViewDev &v = P.views[vi];
            px = pixel_of(v, (int64_t)slot - vbegin[vi], P.tile_w, P.tile_h);
            const CameraRay cam = camera_ray(v, px.px, px.py);
            pt = (float)cam.pt;
            pphi = (float)cam.pphi;
            if constexpr (DRIFT) H0 = (float)cam.H0;
            g = camera_geo(v, cam);
            if (!(v.valid && v.max_steps > 0)) alive = false, st = v.valid ? BHN_RAY_MAX_STEPS : BHN_RAY_INVALID;
        }
        const StepConst &C = sconst[vi];
        for (int it = 0; __any_sync(kFull, alive); ++it) {
            if (it % L.A.interval == 0) {  // warp-wide network evaluation
                float f[8];
                step_features(g, C, pphi, acc.jI, f);
#pragma unroll
                for (int q = 0; q < 8; ++q) f[q] = alive ? (f[q] - N.mu_x[q]) * N.inv_sx[q] : 0.0f;
                const float y = mlp_warp_infer(f, sb, xs, ys);
                mult = __expf(fmaf(N.sig_y, y, N.mu_y) - L.A.margin);
                shrink = 1.0f;
                ++n_net;
            }
            if (!alive) continue;
            if (g.rh < C.r_guard && g.pr < 0.0f) {
                st = BHN_RAY_CAPTURED;
                alive = false;
                continue;
            }
            const float r0 = g.rh + g.rl;
            // the network's multiplier applies to the plain step at the current r
            const float h_plain = fminf(fmaxf(C.hs * r0, C.hmin), C.hmax);
            float h = fminf(fmaxf(fmaxf(mult, L.A.min_scale) * shrink * h_plain, L.A.h_floor), L.A.h_ceil);
            Deriv32 k1, k2;
            rk2_k1(g, C, pt, pphi, k1);
            if constexpr (DRIFT) drift = fmaxf(drift, fabsf(fabsf(k1.H) - H0));
            h = fmaxf(brick_limit(h, g, k1, C, T, P.nr, P.nt, L.A.brick_scale), L.A.h_floor);
            if (crosses_horizon(g, C, h, k1)) {
                st = BHN_RAY_CAPTURED;
                alive = false;
                continue;
            }
            // the Euler and midpoint solutions of an RK2 step differ by h (k2 - k1).
            // The phi difference is weighted by sin(theta) (the angle it subtends):
            // phi is cyclic, so its error does not feed back into the motion, and
            // near the spin axis its coordinate rate ~ 1/sin^2(theta) would
            // otherwise fail every proposal there.
            auto check = [&](const Geo &s0, float hs, const Deriv32 &a1, const Deriv32 &a2) -> float {
                if (!(L.A.check_tol > 0.0f)) return 0.0f;
                const float sth = fabsf(__sinf(s0.th_h));
                return mixed_norm(hs * (a2.r - a1.r), hs * (a2.th - a1.th), sth * hs * (a2.ph - a1.ph),
                                  hs * (a2.pr - a1.pr), hs * (a2.pth - a1.pth), s0, L.A.check_tol);
            };
            Geo y;
            float e;
            if constexpr (SUBSTEPS == 2) {
                // two RK2 steps of h / 2 and one brick segment over both: the form of
                // the controller's accepted solution, without its full-h comparison step
                const float hh = 0.5f * h;
                rk2_stages(g, hh, C, pt, pphi, k1, k2, false);
                e = check(g, hh, k1, k2);
                const Geo ym = geo_advance(g, hh, k2);
                Deriv32 k1b, k2b;
                rk2_stages(ym, hh, C, pt, pphi, k1b, k2b, true);
                e = fmaxf(e, check(ym, hh, k1b, k2b));
                n_eval += 4;
                if (!(e > 1.0f) || L.A.fallback == 2) y = geo_advance(ym, hh, k2b);
            } else {
                rk2_stages(g, h, C, pt, pphi, k1, k2, false);
                n_eval += 2;
                e = check(g, h, k1, k2);
                if (!(e > 1.0f) || L.A.fallback == 2) y = geo_advance(g, h, k2);
            }
            if (e > 1.0f && L.A.fallback == 2) {
                // misprediction, retry form: the step is not taken; this lane takes it
                // again next iteration with a shorter proposal (every lane of the warp
                // runs the same step each iteration, so nothing waits on a fallback
                // path).  After max_attempts tries, or at h_floor, the step is taken.
                ++n_fb;
                if (++fails < L.A.max_attempts && h > L.A.h_floor) {
                    shrink *= fmaxf(0.2f, 0.9f * rsqrtf(e));
                    continue;
                }
            } else if (e > 1.0f) {
                ++n_fb;
                if (L.A.fallback == 0) {  // misprediction: the plain step
                    ++n_eval;
                    h = h_plain;
                    rk2_stages(g, h, C, pt, pphi, k1, k2, false);
                    y = geo_advance(g, h, k2);
                } else {  // misprediction: the step-doubling controller takes this step
                    h = fmaxf(h * fmaxf(0.1f, 0.9f * rsqrtf(e)), L.A.h_floor);
                    float err;
                    unsigned long long n_rej = 0;
                    y = doubling_step(g, h, k1, C, pt, pphi, L.A, err, n_eval, n_rej);
                }
            }
            const float dr = (y.rh - g.rh) + (y.rl - g.rl), dph = (y.ph_h - g.ph_h) + (y.ph_l - g.ph_l);
            const float dph_u = dph > 3.14159f ? dph - kTwoPiH : (dph < -3.14159f ? dph + kTwoPiH : dph);
            brick_segment(T, rec, P.nr, P.nt, P.np, C, g, y, dr, dph_u, acc);
            const bool finite = isfinite(y.rh + y.th_h + y.ph_h + y.pr + y.pth);
            g = y;
            fails = 0;
            ++steps;
            ++n_acc;
            st = terminate(g, C, acc, dr, finite, steps);
            if (st >= 0) alive = false;
        }
        if (slot < total) {
            write_stokes(P.out, (uint32_t)px.out_idx, acc);
            if (P.ray_steps) P.ray_steps[px.out_idx] = steps;
            if (P.ray_status) P.ray_status[px.out_idx] = (uint8_t)st;
            if constexpr (DRIFT) P.ray_drift[px.out_idx] = drift;
        }
        __syncwarp();
    }
    if (L.counters) {
        atomicAdd(&L.counters[0], n_eval);
        atomicAdd(&L.counters[1], n_acc);
        atomicAdd(&L.counters[2], n_fb);
        if (lane == 0) atomicAdd(&L.counters[3], n_net);
    }
}

}  // namespace bhn

// ------------------------------------------------------------ host side
namespace bhn {

static int learn_params(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                        const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                        int64_t scratch_bytes, const bhn_adapt_params *ap, LearnParams &L, int &smem, cudaStream_t s) {
    int rc = check_config(cfg);
    if (rc) return rc;
    if (!ap) return fail(BHN_ERR_VALUE, "adapt params must not be NULL");
    if (!(ap->tol > 0.0f) || !(ap->h_floor > 0.0f) || !(ap->h_ceil >= ap->h_floor) || ap->interval < 1 ||
        ap->max_attempts < 1 || ap->fallback < 0 || ap->fallback > 2 || !(ap->sample_prob >= 0.0f) ||
        !(ap->check_tol >= 0.0f) || !(ap->min_scale > 0.0f) || (ap->substeps != 1 && ap->substeps != 2))
        return fail(BHN_ERR_VALUE, "adapt params: need tol > 0, 0 < h_floor <= h_ceil, check_tol >= 0, min_scale > 0, "
                                   "max_attempts >= 1, substeps 1 or 2");
    if (n_views < 1 || !records || !tables || !out || !scratch) return fail(BHN_ERR_VALUE, "missing buffers or views");
    ScratchLayout SL = scratch_layout(n_views);
    if (scratch_bytes < SL.total) return fail(BHN_ERR_VALUE, "scratch buffer is smaller than bhn_render_scratch_bytes()");
    const int tables_bytes = (int)table_layout(nr, nt, np).total;
    const int64_t sm = smem_bytes(tables_bytes, n_views);
    if (sm > 160 * 1024) return fail(BHN_ERR_VALUE, "brick grids plus views exceed the shared-memory table budget");
    smem = (int)sm;
    char *sc = static_cast<char *>(scratch);
    memset(&L, 0, sizeof L);
    RenderParams &P = L.R;
    P.records = records;
    P.tables = tables;
    P.nr = nr;
    P.nt = nt;
    P.np = np;
    P.n_views = n_views;
    P.views = reinterpret_cast<const ViewDev *>(sc + SL.views);
    P.ray_begin = reinterpret_cast<const int64_t *>(sc + SL.ray_begin);
    P.axis_begin = reinterpret_cast<const int64_t *>(sc + SL.axis_begin);  // unused: these tracers keep the tile order
    P.q = reinterpret_cast<QueueState *>(sc + SL.queue);
    P.stats = reinterpret_cast<bhn_render_stats *>(sc + SL.stats);
    P.out = out;
    P.ray_steps = ray_out ? ray_out->steps : nullptr;
    P.ray_status = ray_out ? ray_out->status : nullptr;
    P.ray_drift = ray_out ? ray_out->h_drift : nullptr;
    P.tile_w = cfg->tile_w;
    P.tile_h = cfg->tile_h;
    P.refill_min = 32;
    P.tables_bytes = tables_bytes;
    L.A.tol = ap->tol;
    L.A.sample_prob = ap->sample_prob;
    L.A.h_floor = ap->h_floor;
    L.A.h_ceil = ap->h_ceil;
    L.A.margin = ap->margin;
    L.A.check_tol = ap->check_tol;
    L.A.brick_scale = ap->brick_scale;
    L.A.min_scale = ap->min_scale;
    L.A.fallback = ap->fallback;
    L.A.interval = ap->interval;
    L.A.max_attempts = ap->max_attempts;
    L.A.seed = ap->seed;
    L.A.substeps = ap->substeps;
    BHN_CUDA_TRY(cudaMemsetAsync(&P.q->next, 0, sizeof(unsigned long long), s));
    return BHN_OK;
}

}  // namespace bhn

extern "C" {

int64_t bhn_mlp_param_count(void) { return kMlpParams; }
int64_t bhn_mlp_blob_bytes(void) { return (int64_t)sizeof(MlpBlob); }

int bhn_mlp_pack(const float *params, const float *h_norm, void *blob, void *stream) {
    if (!params || !h_norm || !blob) return fail(BHN_ERR_VALUE, "params, norm and blob must not be NULL");
    if (reinterpret_cast<uintptr_t>(blob) % 16) return fail(BHN_ERR_VALUE, "blob must be 16-byte aligned");
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, h_norm) == cudaSuccess && attr.type == cudaMemoryTypeDevice)
        return fail(BHN_ERR_VALUE, "h_norm must be host memory");
    cudaGetLastError();  // clear a non-sticky error from the query
    MlpNorm n;
    memcpy(&n, h_norm, 18 * sizeof(float));
    n.pad[0] = n.pad[1] = 0.0f;
    mlp_pack_kernel<<<1, 256, 0, as_stream(stream)>>>(params, n, static_cast<MlpBlob *>(blob));
    BHN_LAUNCH_CHECK("mlp_pack_kernel");
    return BHN_OK;
}

int bhn_mlp_grad(const float *params, const float *samples, const int64_t *index, int64_t first, int64_t count,
                 float *grad, float *loss, void *stream) {
    if (count < 1) return fail(BHN_ERR_VALUE, "batch must contain at least one sample");
    const int smem = (int)train_smem_bytes();
    BHN_CUDA_TRY(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const unsigned blocks = (unsigned)((count + kTrainBlock - 1) / kTrainBlock);
    mlp_grad_kernel<<<blocks, kTrainBlock, smem, as_stream(stream)>>>(params, samples, index, first, count, grad, loss);
    BHN_LAUNCH_CHECK("mlp_grad_kernel");
    return BHN_OK;
}

int bhn_mlp_adam(float *params, float *grad, float *m, float *v, float lr, float beta1, float beta2, float eps,
                 int32_t step, void *stream) {
    if (step < 1) return fail(BHN_ERR_VALUE, "Adam step counts from 1");
    const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
    mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, as_stream(stream)>>>(params, grad, m, v, lr, beta1, beta2,
                                                                             eps, bc1, bc2);
    BHN_LAUNCH_CHECK("mlp_adam_kernel");
    return BHN_OK;
}

int bhn_mlp_infer(const void *blob, const float *features, int64_t n, float *out, void *stream) {
    if (n <= 0) return BHN_OK;
    int64_t blocks = (n + 127) / 128;
    if (blocks > 4096) blocks = 4096;
    mlp_infer_kernel<<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(static_cast<const MlpBlob *>(blob), features, n,
                                                                      out);
    BHN_LAUNCH_CHECK("mlp_infer_kernel");
    return BHN_OK;
}

int bhn_adaptive_launch(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                        const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                        int64_t scratch_bytes, const bhn_adapt_params *ap, float *samples,
                        unsigned long long *sample_count, unsigned long long sample_capacity,
                        unsigned long long *counters, void *stream) {
    cudaStream_t s = as_stream(stream);
    LearnParams L;
    int smem = 0;
    int rc = learn_params(records, tables, nr, nt, np, n_views, cfg, out, ray_out, scratch, scratch_bytes, ap, L, smem, s);
    if (rc) return rc;
    L.samples = samples;
    L.sample_count = sample_count;
    L.sample_capacity = sample_capacity;
    L.counters = counters;
    const int sms = sm_count_current_device();
    auto go = [&](auto kernel) -> int {
        if (smem > 48 * 1024)
            BHN_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kernel<<<sms * cfg->blocks_per_sm, cfg->block_threads, smem, s>>>(L);
        BHN_LAUNCH_CHECK("adaptive_kernel");
        return BHN_OK;
    };
    return L.R.ray_drift ? go(adaptive_kernel<true>) : go(adaptive_kernel<false>);
}

int bhn_learned_launch(const void *records, const void *tables, int32_t nr, int32_t nt, int32_t np, int32_t n_views,
                       const bhn_render_config *cfg, void *out, const bhn_ray_outputs *ray_out, void *scratch,
                       int64_t scratch_bytes, const bhn_adapt_params *ap, const void *blob,
                       unsigned long long *counters, void *stream) {
    if (!blob) return fail(BHN_ERR_VALUE, "network blob must not be NULL");
    cudaStream_t s = as_stream(stream);
    LearnParams L;
    int smem = 0;
    int rc = learn_params(records, tables, nr, nt, np, n_views, cfg, out, ray_out, scratch, scratch_bytes, ap, L, smem, s);
    if (rc) return rc;
    L.blob = static_cast<const MlpBlob *>(blob);
    L.counters = counters;
    const int sms = sm_count_current_device();
    const unsigned blocks = sms * cfg->blocks_per_sm * (cfg->block_threads / 128 > 0 ? cfg->block_threads / 128 : 1);
    auto go = [&](auto kernel) -> int {
        if (smem > 48 * 1024)
            BHN_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        kernel<<<blocks, 128, smem, s>>>(L);
        BHN_LAUNCH_CHECK("learned_kernel");
        return BHN_OK;
    };
    const bool drift = L.R.ray_drift != nullptr;
    if (L.A.substeps == 2) return drift ? go(learned_kernel<true, 2>) : go(learned_kernel<false, 2>);
    return drift ? go(learned_kernel<true, 1>) : go(learned_kernel<false, 1>);
}

}  // extern "C"
