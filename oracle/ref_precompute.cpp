// ref_precompute.cpp -- link-time definitions for the reference's Eigen-based
// precompute functions (code/gpu_planning/cpp/src/planning/chomp_precompute.cpp,
// stomp_precompute.cpp), which need Eigen3 (absent here). The harness never
// calls the reference's host solvers that use them; these restatements exist
// so oracle/_ref/libref_oracle.so links. TEST INFRASTRUCTURE ONLY.
#include <algorithm>
#include <cmath>
#include <vector>

extern "C" void orc_control_cost_R(int T, double dt, double* R);

namespace {

std::vector<double> R64(int T, double dt) {
    std::vector<double> R((size_t)T * T);
    orc_control_cost_R(T, dt, R.data());
    return R;
}

// (R + 1e-8 I)^-1 by Gauss-Jordan with partial pivoting, FP64.
std::vector<double> inv_reg(int T, double dt) {
    std::vector<double> A = R64(T, dt), I((size_t)T * T, 0.0);
    for (int i = 0; i < T; ++i) { A[(size_t)i * T + i] += 1e-8; I[(size_t)i * T + i] = 1.0; }
    for (int c = 0; c < T; ++c) {
        int p = c;
        for (int r = c + 1; r < T; ++r)
            if (std::fabs(A[(size_t)r * T + c]) > std::fabs(A[(size_t)p * T + c])) p = r;
        for (int k = 0; k < T; ++k) { std::swap(A[(size_t)c * T + k], A[(size_t)p * T + k]); std::swap(I[(size_t)c * T + k], I[(size_t)p * T + k]); }
        double d = A[(size_t)c * T + c];
        for (int k = 0; k < T; ++k) { A[(size_t)c * T + k] /= d; I[(size_t)c * T + k] /= d; }
        for (int r = 0; r < T; ++r) {
            if (r == c) continue;
            double f = A[(size_t)r * T + c];
            if (f == 0.0) continue;
            for (int k = 0; k < T; ++k) { A[(size_t)r * T + k] -= f * A[(size_t)c * T + k]; I[(size_t)r * T + k] -= f * I[(size_t)c * T + k]; }
        }
    }
    return I;
}

std::vector<float> to_f(const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); }

}  // namespace

namespace CHOMP {
std::vector<float> compute_control_cost_R(int T, float dt) { return to_f(R64(T, dt)); }
std::vector<float> compute_smoothness_Ainv(int T, float dt) { return to_f(inv_reg(T, dt)); }
}  // namespace CHOMP

namespace STOMP {
std::vector<float> compute_control_cost_R(int T, float dt) { return to_f(R64(T, dt)); }
std::vector<float> compute_cholesky_L(int T, float dt, float noise_scale) {
    std::vector<double> Ri = inv_reg(T, dt);
    double mx = 1e-12;
    for (double v : Ri) mx = std::max(mx, v);
    for (double& v : Ri) v *= (1.0 / T) / mx;
    for (int i = 0; i < T; ++i)
        for (int j = 0; j < i; ++j) {
            double s = 0.5 * (Ri[(size_t)i * T + j] + Ri[(size_t)j * T + i]);
            Ri[(size_t)i * T + j] = Ri[(size_t)j * T + i] = s;
        }
    std::vector<double> L((size_t)T * T, 0.0);
    for (int i = 0; i < T; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = Ri[(size_t)i * T + j];
            for (int k = 0; k < j; ++k) s -= L[(size_t)i * T + k] * L[(size_t)j * T + k];
            L[(size_t)i * T + j] = (i == j) ? std::sqrt(std::max(s, 0.0)) : s / L[(size_t)j * T + j];
        }
    const double sc = noise_scale > 0.0f ? noise_scale : 1.0;
    for (double& v : L) v *= sc;
    return to_f(L);
}
std::vector<float> compute_projection_M(int T, float dt) {
    std::vector<double> Ri = inv_reg(T, dt), M((size_t)T * T);
    for (int j = 0; j < T; ++j) {
        double mx = -1e300;
        for (int i = 0; i < T; ++i) mx = std::max(mx, Ri[(size_t)i * T + j]);
        double sc = (1.0 / T) / std::max(mx, 1e-12);
        for (int i = 0; i < T; ++i) M[(size_t)i * T + j] = Ri[(size_t)i * T + j] * sc;
    }
    return to_f(M);
}
}  // namespace STOMP
