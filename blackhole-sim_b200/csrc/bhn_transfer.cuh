// bhn_transfer.cuh -- the exact constant-coefficient Stokes step (FP64).
//
// python/blackhole_sim/polarized_transfer.py:51-70 solves dS/ds = j - K S over
// one step as the 5x5 augmented exponential
//     [S'; 1] = exp(A ds) [S; 1],   A = [[-K, j], [0, 0]],
// through scipy.linalg.expm.  Here exp(A ds) = [[E, F], [0, 1]] is formed from
// its two blocks by scaling and squaring with a truncated Taylor series
// (Moler & Van Loan, "Nineteen dubious ways to compute the exponential of a
// matrix", 2003, method 3): with X = -K ds / 2^s and ||X||_1 <= 1/4,
//     E_s = sum_{m=0}^{16} X^m / m!,   F_s = sum_{m=0}^{16} X^m y / (m + 1)!,
// y = j ds / 2^s (truncation below 1e-20 relative), then s squarings of the
// block matrix, [[E, F], [0, 1]]^2 = [[E E, E F + F], [0, 1]].

#pragma once

namespace bhn {

// K of native_kernels.py:213-222 / synchrotron.py:82-94 for the 11 COEFF_NAMES
// channels (j_I, j_Q, j_U, j_V, a_I, a_Q, a_U, a_V, r_V, r_Q, r_U).
__host__ __device__ inline void propagation_matrix(const double c[11], double K[4][4]) {
    const double ai = c[4], aq = c[5], au = c[6], av = c[7], rv = c[8], rq = c[9], ru = c[10];
    K[0][0] = ai; K[0][1] = aq;  K[0][2] = au;  K[0][3] = av;
    K[1][0] = aq; K[1][1] = ai;  K[1][2] = rv;  K[1][3] = -ru;
    K[2][0] = au; K[2][1] = -rv; K[2][2] = ai;  K[2][3] = rq;
    K[3][0] = av; K[3][1] = ru;  K[3][2] = -rq; K[3][3] = ai;
}

// S <- E S + F for exp([[-K, j], [0, 0]] ds); ds <= 0 leaves S unchanged
// (polarized_transfer.py:56-57).
__host__ __device__ inline void stokes_step_exact(double S[4], const double c[11], double ds) {
    if (!(ds > 0.0)) return;
    double K[4][4];
    propagation_matrix(c, K);
    double norm = 0.0;  // ||K ds||_1 (largest column sum)
    for (int col = 0; col < 4; ++col) {
        double s = 0.0;
        for (int row = 0; row < 4; ++row) s += fabs(K[row][col]);
        norm = fmax(norm, s * ds);
    }
    int sq = 0;
    double h = ds;
    while (norm > 0.25 && sq < 1100) {  // 2^-1100 scales any finite norm below 1/4
        norm *= 0.5;
        h *= 0.5;
        ++sq;
    }
    double X[4][4], y[4];
    for (int r = 0; r < 4; ++r) {
        for (int k = 0; k < 4; ++k) X[r][k] = -K[r][k] * h;
        y[r] = c[r] * h;
    }
    // Horner: E = I + X (I + X/2 (I + ... (I + X/16))), F = (I + X/2 (I + X/3 (... (I + X/17)))) y
    double E[4][4], F[4];
    for (int r = 0; r < 4; ++r) {
        for (int k = 0; k < 4; ++k) E[r][k] = r == k ? 1.0 : 0.0;
        F[r] = y[r];
    }
    for (int m = 16; m >= 1; --m) {
        double T[4][4], Fn[4];
        const double inv_e = 1.0 / m, inv_f = 1.0 / (m + 1);
        for (int r = 0; r < 4; ++r) {
            double fv = 0.0;
            for (int k = 0; k < 4; ++k) {
                double t = 0.0;
                for (int l = 0; l < 4; ++l) t += X[r][l] * E[l][k];
                T[r][k] = (r == k ? 1.0 : 0.0) + t * inv_e;
                fv += X[r][k] * F[k];
            }
            Fn[r] = y[r] + fv * inv_f;
        }
        for (int r = 0; r < 4; ++r) {
            for (int k = 0; k < 4; ++k) E[r][k] = T[r][k];
            F[r] = Fn[r];
        }
    }
    for (int it = 0; it < sq; ++it) {
        double E2[4][4], F2[4];
        for (int r = 0; r < 4; ++r) {
            double fv = 0.0;
            for (int k = 0; k < 4; ++k) {
                double t = 0.0;
                for (int l = 0; l < 4; ++l) t += E[r][l] * E[l][k];
                E2[r][k] = t;
                fv += E[r][k] * F[k];
            }
            F2[r] = fv + F[r];
        }
        for (int r = 0; r < 4; ++r) {
            for (int k = 0; k < 4; ++k) E[r][k] = E2[r][k];
            F[r] = F2[r];
        }
    }
    double out[4];
    for (int r = 0; r < 4; ++r) {
        double v = F[r];
        for (int k = 0; k < 4; ++k) v += E[r][k] * S[k];
        out[r] = v;
    }
    for (int r = 0; r < 4; ++r) S[r] = out[r];
}

}  // namespace bhn
