// ref_precompute.cpp -- FP32 restatements of the reference's Eigen-based
// precompute functions (code/gpu_planning/cpp/src/planning/chomp_precompute.cpp:
// 20-63, stomp_precompute.cpp:24-114). Eigen3 is absent here, so the harness
// links these in their place, and the reference's host solvers that the
// harness runs (CHOMP::solve_runtime_scene, chomp.cu:421-423;
// STOMP::solve_runtime_scene, stomp.cu:681-696) DO call them: every
// "reference solver" result is the reference's solver code over this
// restatement, not over Eigen itself. TEST INFRASTRUCTURE ONLY.
//
// The arithmetic follows what the reference asks Eigen for, in FP32
// (Eigen::MatrixXf) throughout:
//   R       = dt * (A^T A), A the 5-point acceleration operator on a grid
//             padded by 6 each side, central T x T block (an FP32 product);
//   R + 1e-8 I in FP32 (the shift is below one ulp of R's diagonal, as in
//             the reference's FP32 sum);
//   inverse() of a dynamic-size matrix = Eigen's PartialPivLU: LU with row
//             partial pivoting (right-looking elimination), then a forward
//             and a back substitution per column of the permuted identity;
//   LLT     = Cholesky factor, lower, computed column by column.
// Eigen blocks and vectorises these, so its summation order differs and its
// bits can differ in the last places; the algorithms and the precision are
// the reference's. Restated from the published algorithms, no Eigen source.
#include <algorithm>
#include <cmath>
#include <vector>

namespace {

constexpr int kPad = 6;

// Row-major FP32 matrices.
std::vector<float> build_R32(int T, float dt) {
    const int Np = T + 2 * kPad;
    const float inv_dt2 = 1.0f / (dt * dt);
    const float coeff[7] = {0.0f, -1.0f / 12.0f, 16.0f / 12.0f, -30.0f / 12.0f, 16.0f / 12.0f, -1.0f / 12.0f, 0.0f};
    std::vector<float> A((size_t)Np * Np, 0.0f);
    for (int i = 0; i < Np; ++i)
        for (int j = -3; j <= 3; ++j) {
            const int idx = i + j;
            if (idx >= 0 && idx < Np) A[(size_t)i * Np + idx] = inv_dt2 * coeff[j + 3];
        }
    std::vector<float> R((size_t)T * T);
    for (int a = 0; a < T; ++a)
        for (int b = 0; b < T; ++b) {
            float acc = 0.0f;   // (A^T A)(a+6, b+6), FP32 accumulation
            for (int k = 0; k < Np; ++k) acc += A[(size_t)k * Np + a + kPad] * A[(size_t)k * Np + b + kPad];
            R[(size_t)a * T + b] = dt * acc;
        }
    return R;
}

// (R + 1e-8 I)^-1 through an FP32 LU factorisation with partial pivoting.
std::vector<float> inverse_pplu(std::vector<float> M, int T) {
    std::vector<int> perm(T);
    for (int i = 0; i < T; ++i) perm[i] = i;
    for (int k = 0; k < T; ++k) {
        int p = k;
        for (int i = k + 1; i < T; ++i)
            if (std::fabs(M[(size_t)i * T + k]) > std::fabs(M[(size_t)p * T + k])) p = i;
        if (p != k) {
            for (int j = 0; j < T; ++j) std::swap(M[(size_t)k * T + j], M[(size_t)p * T + j]);
            std::swap(perm[k], perm[p]);
        }
        const float piv = M[(size_t)k * T + k];
        for (int i = k + 1; i < T; ++i) {
            const float l = M[(size_t)i * T + k] / piv;
            M[(size_t)i * T + k] = l;
            for (int j = k + 1; j < T; ++j) M[(size_t)i * T + j] -= l * M[(size_t)k * T + j];
        }
    }
    std::vector<float> X((size_t)T * T), y(T);
    for (int c = 0; c < T; ++c) {
        for (int i = 0; i < T; ++i) {   // L y = P e_c (unit lower)
            float s = perm[i] == c ? 1.0f : 0.0f;
            for (int k = 0; k < i; ++k) s -= M[(size_t)i * T + k] * y[k];
            y[i] = s;
        }
        for (int i = T - 1; i >= 0; --i) {   // U x = y
            float s = y[i];
            for (int k = i + 1; k < T; ++k) s -= M[(size_t)i * T + k] * X[(size_t)k * T + c];
            X[(size_t)i * T + c] = s / M[(size_t)i * T + i];
        }
    }
    return X;
}

std::vector<float> inv_reg32(int T, float dt) {
    std::vector<float> R = build_R32(T, dt);
    for (int i = 0; i < T; ++i) R[(size_t)i * T + i] += 1.0e-8f;
    return inverse_pplu(R, T);
}

}  // namespace

namespace CHOMP {
std::vector<float> compute_control_cost_R(int T, float dt) { return build_R32(T, dt); }
std::vector<float> compute_smoothness_Ainv(int T, float dt) { return inv_reg32(T, dt); }
}  // namespace CHOMP

namespace STOMP {
std::vector<float> compute_control_cost_R(int T, float dt) { return build_R32(T, dt); }

std::vector<float> compute_cholesky_L(int T, float dt, float noise_scale) {
    std::vector<float> Ri = inv_reg32(T, dt);
    float mx = Ri[0];
    for (float v : Ri) mx = std::max(mx, v);
    mx = std::max(mx, 1.0e-12f);
    const float sc = (1.0f / (float)T) / mx;
    for (float& v : Ri) v *= sc;
    std::vector<float> S((size_t)T * T);   // 0.5 (Ri + Ri^T)
    for (int i = 0; i < T; ++i)
        for (int j = 0; j < T; ++j) S[(size_t)i * T + j] = 0.5f * (Ri[(size_t)i * T + j] + Ri[(size_t)j * T + i]);
    std::vector<float> L((size_t)T * T, 0.0f);   // LLT, lower, column by column
    for (int j = 0; j < T; ++j) {
        float d = S[(size_t)j * T + j];
        for (int k = 0; k < j; ++k) d -= L[(size_t)j * T + k] * L[(size_t)j * T + k];
        const float ljj = std::sqrt(std::max(d, 0.0f));
        L[(size_t)j * T + j] = ljj;
        for (int i = j + 1; i < T; ++i) {
            float s = S[(size_t)i * T + j];
            for (int k = 0; k < j; ++k) s -= L[(size_t)i * T + k] * L[(size_t)j * T + k];
            L[(size_t)i * T + j] = ljj > 0.0f ? s / ljj : 0.0f;
        }
    }
    const float s = noise_scale > 0.0f ? noise_scale : 1.0f;
    for (float& v : L) v *= s;
    return L;
}

std::vector<float> compute_projection_M(int T, float dt) {
    const std::vector<float> Ri = inv_reg32(T, dt);
    std::vector<float> M((size_t)T * T);
    const float inv_T = 1.0f / (float)T;
    for (int j = 0; j < T; ++j) {
        float col_max = Ri[j];
        for (int i = 0; i < T; ++i) col_max = std::max(col_max, Ri[(size_t)i * T + j]);
        const float sc = inv_T / std::max(col_max, 1.0e-12f);
        for (int i = 0; i < T; ++i) M[(size_t)i * T + j] = Ri[(size_t)i * T + j] * sc;
    }
    return M;
}
}  // namespace STOMP
