// ps_stomp.cu -- batched STOMP optimiser loop on the device.
//
// The reference runs one STOMP request at a time (STOMP::solve_runtime_scene,
// stomp.cu:565-965): per iteration about 15 launches over dense T x T
// matrices (noise L z, control cost R theta, projection M delta), cuRAND
// XORWOW states per (rollout, d, t), a single-thread top-k, full copies of the
// rollout population into "previous" buffers, then the same host
// bookkeeping as CHOMP with a D*T readback for the validity densification.
//
// Here B requests advance together and every operator is banded:
//   * R + 1e-8 I = Lb Lb^T (bandwidth 4, FP64, once per call). R is
//     persymmetric (J R J = R), so the lower Cholesky factor of
//     c (R + 1e-8 I)^-1 is sqrt(c) J Lb^-T J: the noise L z is one banded
//     back substitution per (request, rollout, DoF) instead of a T x T
//     product; M delta = (R + 1e-8 I)^-1 (s .* delta) is one banded solve
//     with the column scales s of stomp_precompute.cpp:70-94;
//   * the normal variates come from a counter-based generator (Philox4x32-10
//     with Box-Muller), so no generator state is stored or copied;
//   * rollout rows are laid out rollout-major over the requests
//     (row = r * B + b) so that the fresh rows of all requests form one
//     contiguous range for the cost kernel; the rollout population is double
//     buffered by iteration parity instead of copied;
//   * control costs, per-rollout totals, the exponentiated weights and the
//     weighted noise run as three small kernels over all requests;
//   * validity and bookkeeping are shared with the CHOMP loop
//     (ps_optloop.cuh).
#include <algorithm>
#include <cstring>

#include "ps_costwarp.cuh"
#include "ps_optloop.cuh"

namespace ps {
namespace {

// ---- counter-based normal variates ---------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): ten rounds of two 32x32->64 multiplies with the
// published multipliers and Weyl key increments.
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// The top 24 bits as a float strictly inside (0, 1).
__device__ __forceinline__ float unit_open(uint32_t x) {
    return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// Box-Muller: two uniforms to two independent standard normals.
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& z0, float& z1) {
    const float r = sqrtf(-2.0f * logf(unit_open(a)));
    float s, c;
    sincospif(2.0f * unit_open(b), &s, &c);
    z0 = r * c;
    z1 = r * s;
}

// x <- (Lb^T)^-1 x for the banded factor of opt_band_kernel (the second half
// of band_solve).
__device__ __forceinline__ void band_back(const double* Ls, double* x, int T) { band_backward(Ls, x, T); }

// Column scales of M and the noise amplitude (stomp_precompute.cpp:46-94):
// with Rinv = (R + 1e-8 I)^-1, s_j = (1/T) / max_i Rinv(i, j) and
// sqrt_c = noise_scale * sqrt((1/T) / max_ij Rinv(i, j)). One thread per
// column of Rinv (a banded solve of e_j into scratch [T][T]). FP64.
__global__ void stomp_setup_kernel(int T, const double* __restrict__ band, double* __restrict__ scratch,
                                   double* __restrict__ colscale, double* __restrict__ amp, float noise_scale) {
    __shared__ double red[256];
    double gmax = -INFINITY;
    for (int j = threadIdx.x; j < T; j += blockDim.x) {
        double* x = scratch + (size_t)j * T;
        for (int i = 0; i < T; ++i) x[i] = (i == j) ? 1.0 : 0.0;
        band_solve(band, x, T);
        double mx = -INFINITY;
        for (int i = 0; i < T; ++i) mx = fmax(mx, x[i]);
        colscale[j] = (1.0 / T) / fmax(mx, 1.0e-12);
        gmax = fmax(gmax, mx);
    }
    red[threadIdx.x] = gmax;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double sc = noise_scale > 0.0f ? (double)noise_scale : 1.0;
        amp[0] = sc * sqrt((1.0 / T) / fmax(red[0], 1.0e-12));
    }
}

__device__ __forceinline__ bool stomp_active(const OptState* state, const uint8_t* done, int b) {
    return !done[b] && state[b].step >= 1;
}

// Per request: the num_rollouts_old lowest row totals of the previous
// iteration, by the reference's selection (stomp.cu:133-152: repeated
// first-minimum scan, each pick masked with 3e38). Thread 0; the totals
// staged in shared memory.
__global__ void stomp_topk_kernel(const float* __restrict__ tot_prev, int* __restrict__ topk, int R, int Ro, int B,
                                  const OptState* __restrict__ state, const uint8_t* __restrict__ done) {
    extern __shared__ float cc[];   // [R]
    const int b = blockIdx.x;
    if (Ro == 0 || !stomp_active(state, done, b) || state[b].step == 1) return;
    for (int r = threadIdx.x; r < R; r += blockDim.x) cc[r] = tot_prev[(size_t)r * B + b];
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int k = 0; k < Ro; ++k) {
        int bi = 0;
        float bc = cc[0];
        for (int i = 1; i < R; ++i)
            if (cc[i] < bc) {
                bc = cc[i];
                bi = i;
            }
        topk[(size_t)b * Ro + k] = bi;
        cc[bi] = 3.0e38f;
    }
}

// One block per group of kg rollouts r of request b, row = r * B + b:
//   r < Rn (or < Rn + Ro on the first iteration): fresh rollout
//     clamp(theta + L z), endpoints pinned (stomp.cu:96-130);
//   Rn <= r < Rn + Ro afterwards: the previous iteration's reuse row, noise
//     recomputed against the current optimum (stomp.cu:155-177);
//   r = R - 1: the optimum itself with its state cost (stomp.cu:180-203).
// Also writes the cost kernel's skip byte of rows < Rn + Ro. The banded back
// substitution is sequential over t, one thread per (rollout, DoF) chain:
// with kg rollouts per block, kg * D threads run chains at once instead of
// D while the rest of the block waits at the barrier.
__global__ void stomp_rollouts_kernel(const float* __restrict__ theta, int B, int T, int D, int Rn, int Ro, int kg,
                                      const double* __restrict__ band, const double* __restrict__ amp,
                                      uint32_t key0, uint32_t key1, const float* __restrict__ lower,
                                      const float* __restrict__ upper, float* __restrict__ roll_cur,
                                      const float* __restrict__ roll_prev, float* __restrict__ noise,
                                      float* __restrict__ sc_cur, const float* __restrict__ sc_prev,
                                      const float* __restrict__ opt_sc, const int* __restrict__ topk,
                                      uint8_t* __restrict__ skip, const OptState* __restrict__ state,
                                      const uint8_t* __restrict__ done) {
    // shared: the band factor [T][5], then one chain of T + 1 doubles per
    // (rollout g, DoF d) in reversed order, zs[(g * D + d) * (T + 1) + (T - 1 - t)] = z_t;
    // the odd stride puts the chains that the threads walk side by side in
    // different banks
    extern __shared__ double sm_ro[];
    double* Ls = sm_ro;
    double* zs = sm_ro + (size_t)T * 5;
    const int S = T + 1;
    const int b = blockIdx.y, r0 = blockIdx.x * kg;
    const int R = Rn + Ro + 1;
    const int ng = min(kg, R - r0);
    const bool active = stomp_active(state, done, b);
    const int step = state[b].step;
    const bool init = step == 1;
    for (int g = threadIdx.x; g < ng; g += blockDim.x) {
        const int r = r0 + g;
        if (r < Rn + Ro) skip[(size_t)r * B + b] = (!active || (r >= Rn && !init)) ? 1 : 0;
    }
    if (!active) return;
    const float* th = theta + (size_t)b * T * D;
    // fresh rollouts of the group: r < Rn, or r < Rn + Ro on the first iteration
    auto fresh = [&](int r) { return r < Rn || (init && r < Rn + Ro); };
    // copies: the optimum row and the reuse rows
    for (int g = 0; g < ng; ++g) {
        const int r = r0 + g;
        if (fresh(r)) continue;
        const size_t row = (size_t)r * B + b;
        float* ro = roll_cur + row * T * D;
        float* no = noise + row * T * D;
        if (r == R - 1) {
            for (int i = threadIdx.x; i < T * D; i += blockDim.x) {
                ro[i] = th[i];
                no[i] = 0.0f;
            }
            for (int t = threadIdx.x; t < T; t += blockDim.x) sc_cur[row * T + t] = opt_sc[(size_t)b * T + t];
        } else {
            const size_t srow = (size_t)topk[(size_t)b * Ro + (r - Rn)] * B + b;
            const float* src = roll_prev + srow * T * D;
            for (int i = threadIdx.x; i < T * D; i += blockDim.x) {
                const float v = src[i];
                ro[i] = v;
                no[i] = v - th[i];
            }
            for (int t = threadIdx.x; t < T; t += blockDim.x) sc_cur[row * T + t] = sc_prev[srow * T + t];
        }
    }
    int nf = 0;   // fresh rollouts come first in a group (r ascending)
    while (nf < ng && fresh(r0 + nf)) ++nf;
    if (nf == 0) return;   // uniform over the block
    for (int i = threadIdx.x; i < T * 5; i += blockDim.x) Ls[i] = band[i];
    const int nk = (T + 3) / 4;
    for (int it = threadIdx.x; it < nf * D * nk; it += blockDim.x) {
        const int gd = it / nk, k = it - gd * nk;
        const int g = gd / D, d = gd - g * D;
        const U4 o = philox4x32_10(U4{(uint32_t)k, (uint32_t)((r0 + g) * D + d), (uint32_t)step, 0u}, key0, key1);
        float z[4];
        box_muller(o.x, o.y, z[0], z[1]);
        box_muller(o.z, o.w, z[2], z[3]);
        for (int j = 0; j < 4; ++j) {
            const int t = 4 * k + j;
            if (t < T) zs[gd * S + (T - 1 - t)] = (double)z[j];
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nf * D; c += blockDim.x) band_back(Ls, zs + (size_t)c * S, T);
    __syncthreads();
    const double a = amp[0];
    for (int i = threadIdx.x; i < nf * T * D; i += blockDim.x) {
        const int g = i / (T * D), e = i - g * (T * D);
        const int t = e / D, d = e - t * D;
        const float n = (t == 0 || t == T - 1) ? 0.0f : (float)(a * zs[(g * D + d) * S + (T - 1 - t)]);
        const float base = th[e];
        const float v = fmaxf(lower[d], fminf(upper[d], base + n));
        const size_t row = (size_t)(r0 + g) * B + b;
        roll_cur[row * T * D + e] = v;
        noise[row * T * D + e] = v - base;
    }
}

// One block per (rollout, request): control cost per (t, d),
// w_c theta_t (R theta)_t with R theta as two 5-tap stencils over the
// 6-padded rollout (stomp.cu:257-275), and the row total
// sum_t (state_t + sum_d control_t,d) (stomp.cu:283-308).
__global__ void stomp_row_totals_kernel(const float* __restrict__ roll_cur, const float* __restrict__ sc_cur,
                                        float* __restrict__ ctrl, float* __restrict__ tot_cur, int B, int T, int D,
                                        float w_c, float dt, const OptState* __restrict__ state,
                                        const uint8_t* __restrict__ done) {
    extern __shared__ float sh[];   // xs [(T + 12) D], ac [(T + 12) D], red [blockDim]
    const int r = blockIdx.x, b = blockIdx.y;
    if (!stomp_active(state, done, b)) return;
    const int Np = T + 12;
    float* xs = sh;
    float* ac = xs + (size_t)Np * D;
    float* red = ac + (size_t)Np * D;
    const size_t row = (size_t)r * B + b;
    const float* x = roll_cur + row * T * D;
    for (int i = threadIdx.x; i < Np * D; i += blockDim.x) {
        const int k = i / D, d = i - k * D, t = k - 6;
        xs[i] = (t >= 0 && t < T) ? x[(size_t)t * D + d] : 0.0f;
    }
    __syncthreads();
    const float c1 = -1.0f / 12.0f, c2 = 16.0f / 12.0f, c3 = -30.0f / 12.0f, inv_dt2 = 1.0f / (dt * dt);
    for (int i = threadIdx.x; i < Np * D; i += blockDim.x) {
        const int k = i / D, d = i - k * D;
        auto at = [&](int kk) { return (kk >= 0 && kk < Np) ? xs[kk * D + d] : 0.0f; };
        ac[i] = (c1 * (at(k - 2) + at(k + 2)) + c2 * (at(k - 1) + at(k + 1)) + c3 * at(k)) * inv_dt2;
    }
    __syncthreads();
    float part = 0.0f;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const int k = t + 6;
        float rowsum = sc_cur[row * T + t];
        for (int d = 0; d < D; ++d) {
            const float rt = (c1 * (ac[(k - 2) * D + d] + ac[(k + 2) * D + d]) +
                              c2 * (ac[(k - 1) * D + d] + ac[(k + 1) * D + d]) + c3 * ac[k * D + d]) * inv_dt2 * dt;
            const float c = w_c * xs[k * D + d] * rt;
            ctrl[row * T * D + (size_t)t * D + d] = c;
            rowsum += c;
        }
        part += rowsum;
    }
    red[threadIdx.x] = part;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) tot_cur[row] = red[0];
}

// One thread per (request, t, d): over the R rollouts, cost
// c_r = state_r,t + control_r,t,d, weights p_r = exp(-h (c_r - min) /
// max(max - min, 1e-8)) / max(sum, 1e-12) (stomp.cu:314-355), and the
// weighted noise delta = sum_r p_r noise_r, 0 at the endpoints
// (stomp.cu:360-385).
__global__ void stomp_weights_kernel(const float* __restrict__ sc_cur, const float* __restrict__ ctrl,
                                     const float* __restrict__ noise, float* __restrict__ delta, int B, int T, int D,
                                     int R, float h, const OptState* __restrict__ state,
                                     const uint8_t* __restrict__ done) {
    const long long n = (long long)B * T * D;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(idx / ((long long)T * D));
        const int rem = (int)(idx - (long long)b * T * D);
        const int t = rem / D;
        if (!stomp_active(state, done, b)) continue;
        auto cost = [&](int r) {
            const size_t row = (size_t)r * B + b;
            return sc_cur[row * T + t] + ctrl[row * T * D + rem];
        };
        // the rollouts go in batches of 8 whose loads are all issued before
        // their values are used, so that each thread keeps 16 or 24 loads in
        // flight (the kernel waited on one load at a time); the min/max, the
        // sum and the weighted noise still run in rollout order
        constexpr int kB = 8;
        float mn = cost(0), mx = mn;
        int r = 1;
        for (; r + kB <= R; r += kB) {
            float c[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) c[k] = cost(r + k);
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                mn = fminf(mn, c[k]);
                mx = fmaxf(mx, c[k]);
            }
        }
        for (; r < R; ++r) {
            const float c = cost(r);
            mn = fminf(mn, c);
            mx = fmaxf(mx, c);
        }
        const float denom = fmaxf(mx - mn, 1.0e-8f);
        float sum = 0.0f;
        for (r = 0; r + kB <= R; r += kB) {
            float c[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) c[k] = cost(r + k);
#pragma unroll
            for (int k = 0; k < kB; ++k) sum += expf(-h * (c[k] - mn) / denom);
        }
        for (; r < R; ++r) sum += expf(-h * (cost(r) - mn) / denom);
        sum = fmaxf(sum, 1.0e-12f);
        float acc = 0.0f;
        for (r = 0; r + kB <= R; r += kB) {
            float c[kB], z[kB];
#pragma unroll
            for (int k = 0; k < kB; ++k) {
                c[k] = cost(r + k);
                z[k] = noise[((size_t)(r + k) * B + b) * T * D + rem];
            }
#pragma unroll
            for (int k = 0; k < kB; ++k) acc += z[k] * (expf(-h * (c[k] - mn) / denom) / sum);
        }
        for (; r < R; ++r) {
            const float p = expf(-h * (cost(r) - mn) / denom) / sum;
            acc += noise[((size_t)r * B + b) * T * D + rem] * p;
        }
        delta[idx] = (t == 0 || t == T - 1) ? 0.0f : acc;
    }
}

// One block per (request, DoF): theta_d += M delta_d on the interior
// waypoints, M delta = (R + 1e-8 I)^-1 (s .* delta) (stomp.cu:390-413),
// FP64 banded solve in thread 0. The optimum takes the update
// unconditionally (stomp.cu:415-466).
__global__ void stomp_project_kernel(float* __restrict__ theta, const float* __restrict__ delta,
                                     const double* __restrict__ band, const double* __restrict__ colscale, int B,
                                     int T, int D, const OptState* __restrict__ state,
                                     const uint8_t* __restrict__ done) {
    extern __shared__ double shp[];   // x [T], Ls [5 T]
    const int b = blockIdx.x / D, d = blockIdx.x % D;
    if (!stomp_active(state, done, b)) return;
    double* x = shp;
    double* Ls = x + T;
    for (int k = threadIdx.x; k < 5 * T; k += blockDim.x) Ls[k] = band[k];
    for (int t = threadIdx.x; t < T; t += blockDim.x)
        x[t] = colscale[t] * (double)delta[((size_t)b * T + t) * D + d];
    __syncthreads();
    if (threadIdx.x == 0) band_solve(Ls, x, T);
    __syncthreads();
    float* col = theta + (size_t)b * T * D + d;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        if (t == 0 || t == T - 1) continue;
        col[(size_t)t * D] = col[(size_t)t * D] + (float)x[t];
    }
}

// One block per request: total = sum of the optimum's state costs +
// w_c sum_d theta_d^T R theta_d (stomp.cu:466-500), then the shared
// bookkeeping.
__global__ void stomp_bookkeep_kernel(const float* __restrict__ theta, const float* __restrict__ opt_sc,
                                      const uint8_t* __restrict__ seg_valid, const uint8_t* __restrict__ wp_hit,
                                      int T, int D, ps_cost_params P, int n_iter, float conv_eps,
                                      float time_limit_ms, const unsigned long long* __restrict__ t0,
                                      OptState* __restrict__ state, uint8_t* __restrict__ done,
                                      float* __restrict__ best, int* __restrict__ n_done) {
    extern __shared__ float sh[];   // traj_smooth_block: 2 (T + 12) + blockDim
    const int b = blockIdx.x;
    if (done[b]) return;
    const float* th = theta + (size_t)b * T * D;
    const float total = traj_smooth_block([&](int t, int d) { return th[(size_t)t * D + d]; },
                                          [&](int, int, float) {},
                                          [&](int t) { return opt_sc[(size_t)b * T + t]; }, T, D, P, false, sh);
    opt_bookkeep_block(b, th, total, seg_valid, wp_hit, T, D, n_iter, conv_eps, time_limit_ms, t0, state, done, best,
                       n_done);
}

struct StompBufs {
    OptBufs o;
    float *roll[2], *noise, *ctrl, *sc[2], *tot[2], *delta, *opt_sc;
    uint8_t* skip;
    int* topk;
    double *colscale, *amp, *scratch;
    size_t off_roll[2], off_noise, off_sc[2], off_tot[2], off_topk;
};

size_t stomp_layout(int B, int T, int D, int Rn, int Ro, StompBufs* out, void* base) {
    StompBufs w;
    Carver c{reinterpret_cast<unsigned char*>(base)};
    const size_t Bq = (size_t)std::max(B, 1), Tq = (size_t)std::max(T, 1);
    const size_t rows = (size_t)(Rn + Ro + 1) * Bq;
    opt_carve(c, B, T, D, w.o);
    for (int p = 0; p < 2; ++p) {
        w.off_roll[p] = c.off;
        w.roll[p] = c.take<float>(4 * rows * Tq * D);
    }
    w.off_noise = c.off;
    w.noise = c.take<float>(4 * rows * Tq * D);
    w.ctrl = c.take<float>(4 * rows * Tq * D);
    for (int p = 0; p < 2; ++p) {
        w.off_sc[p] = c.off;
        w.sc[p] = c.take<float>(4 * rows * Tq);
    }
    for (int p = 0; p < 2; ++p) {
        w.off_tot[p] = c.off;
        w.tot[p] = c.take<float>(4 * rows);
    }
    w.delta = c.take<float>(4 * Bq * Tq * D);
    w.opt_sc = c.take<float>(4 * Bq * Tq);
    w.skip = c.take<uint8_t>((size_t)(Rn + Ro) * Bq);
    w.off_topk = c.off;
    w.topk = c.take<int>(4 * Bq * (size_t)std::max(Ro, 1));
    w.colscale = c.take<double>(8 * Tq);
    w.amp = c.take<double>(8);
    w.scratch = c.take<double>(8 * Tq * Tq);
    if (out) *out = w;
    return c.off;
}

int check_stomp_args(const ps_model* m, int B, int T, const ps_stomp_params* P) {
    if (!m || !P) return set_error(PS_EINVAL, "model / params is NULL");
    if (B < 0) return set_error(PS_EINVAL, "B < 0");
    if (T < 2 || T > kOptMaxT) return set_error(PS_EINVAL, "T must be in [2, 1024]");
    if (P->num_rollouts_new < 1 || P->num_rollouts_old < 0 || P->num_rollouts_new + P->num_rollouts_old + 1 > 1024)
        return set_error(PS_EINVAL, "rollout counts out of range");
    if (P->num_iterations < 0 || P->num_iterations_after_valid < 0)
        return set_error(PS_EINVAL, "negative iteration count");
    if (!(P->delta_t > 0.0f)) return set_error(PS_EINVAL, "delta_t must be > 0");
    const long long rows = (long long)(P->num_rollouts_new + P->num_rollouts_old + 1) * B;
    if (rows * T >= (1ll << 31)) return set_error(PS_EINVAL, "rollouts * B * T exceeds 2^31");
    return PS_OK;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" size_t ps_stomp_workspace_bytes(const ps_model* m, int B, int T, const ps_stomp_params* P) {
    if (check_stomp_args(m, B, T, P) != PS_OK) {
        clear_error();
        return 0;
    }
    return stomp_layout(B, T, m->info.n_dof, P->num_rollouts_new, P->num_rollouts_old, nullptr, nullptr);
}

extern "C" int ps_stomp_workspace_layout(const ps_model* m, int B, int T, const ps_stomp_params* P,
                                         ps_stomp_layout* out) {
    clear_error();
    if (int rc = check_stomp_args(m, B, T, P)) return rc;
    if (!out) return set_error(PS_EINVAL, "out is NULL");
    StompBufs w;
    stomp_layout(B, T, m->info.n_dof, P->num_rollouts_new, P->num_rollouts_old, &w, nullptr);
    out->rows = P->num_rollouts_new + P->num_rollouts_old + 1;
    for (int p = 0; p < 2; ++p) {
        out->rollouts[p] = w.off_roll[p];
        out->state_cost[p] = w.off_sc[p];
        out->row_total[p] = w.off_tot[p];
    }
    out->noise = w.off_noise;
    out->reuse_index = w.off_topk;
    return PS_OK;
}

extern "C" int ps_stomp_optimize(const ps_model* m, const ps_scene_view* scene, float* theta, int B, int T,
                                 const ps_stomp_params* P, float* best, uint8_t* solved, int* iterations,
                                 float* best_cost, void* workspace, size_t workspace_bytes, void* stream) {
    PS_NVTX("ps_stomp_optimize");
    clear_error();
    if (int rc = check_stomp_args(m, B, T, P)) return rc;
    if (int rc = validate_scene(m, scene)) return rc;
    if (B == 0) return PS_OK;
    if (!theta || !best || !solved || !iterations || !best_cost) return set_error(PS_EINVAL, "NULL output buffer");
    if (m->info.n_joints > 255) return set_error(PS_EINVAL, "too many joints");
    const int D = m->info.n_dof;
    const int Rn = P->num_rollouts_new, Ro = P->num_rollouts_old, R = Rn + Ro + 1;
    if (!workspace || workspace_bytes < ps_stomp_workspace_bytes(m, B, T, P))
        return set_error(PS_EINVAL, "workspace missing or smaller than ps_stomp_workspace_bytes");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return set_error(PS_EINVAL, "workspace not 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    StompBufs w;
    stomp_layout(B, T, D, Rn, Ro, &w, workspace);
    const OptBufs& o = w.o;

    ps_cost_params cp{};   // state cost: the summed hinge only (stomp.cu:206-245)
    cp.collision_cost_weight = P->collision_cost_weight;
    cp.world_margin = P->world_margin;
    cp.self_margin = P->self_margin;
    cp.include_self = P->include_self;
    cp.smoothness_weight = 0.0f;
    cp.delta_t = P->delta_t;
    cp.layout = PS_LAYOUT_BTD;
    ps_cost_params cp_total = cp;
    cp_total.smoothness_weight = P->control_cost_weight;
    const uint32_t key0 = (uint32_t)(P->seed & 0xffffffffull), key1 = (uint32_t)(P->seed >> 32);

    opt_band_kernel<<<1, 1, 0, s>>>(T, P->delta_t, o.band);
    stomp_setup_kernel<<<1, 256, 0, s>>>(T, o.band, w.scratch, w.colscale, w.amp, P->noise_scale);
    opt_init_kernel<<<(B + 127) / 128, 128, 0, s>>>(o.state, o.done, B, P->num_iterations_after_valid, o.n_done, o.t0);
    PS_TRY_CUDA(cudaGetLastError());

    // rollouts per block of the rollouts kernel: up to 8, within 96 KiB of
    // shared memory and 128 chains (threads)
    const size_t ro_one = sizeof(double) * (size_t)D * (T + 1), ro_band = sizeof(double) * 5 * (size_t)T;
    const int ro_kg = (int)std::max<size_t>(1, std::min<size_t>({(size_t)8, (size_t)(96 * 1024) / ro_one,
                                                                 (size_t)(128 / std::max(D, 1))}));
    const size_t ro_smem = ro_band + ro_one * ro_kg;
    const int tot_threads = 128;
    const size_t tot_smem = sizeof(float) * ((size_t)2 * (T + 12) * D + tot_threads);
    const size_t pj_smem = sizeof(double) * 6 * (size_t)T;
    const int bk_threads = 128;
    const size_t bk_smem = (size_t)(2 * (T + 12) + bk_threads) * sizeof(float);
    auto big = [](auto kernel, size_t bytes) -> int {
        if (bytes > 48 * 1024)
            PS_TRY_CUDA(allow_smem((const void*)kernel, bytes));
        return PS_OK;
    };
    if (int rc = big(stomp_rollouts_kernel, ro_smem)) return rc;
    if (int rc = big(stomp_row_totals_kernel, tot_smem)) return rc;
    if (int rc = big(stomp_project_kernel, pj_smem)) return rc;
    if (int rc = big(stomp_bookkeep_kernel, bk_smem)) return rc;
    if (int rc = big(stomp_topk_kernel, sizeof(float) * (size_t)R)) return rc;
    const long long n_w = (long long)B * T * D;
    const int w_grid = (int)std::min<long long>((n_w + 255) / 256, (long long)sm_count() * 16);

    // One iteration at chunk position i (parity i & 1; a chunk has an even
    // length, so the parity is the iteration's own): a request at step 0 is
    // only evaluated (the seed); from step 1 on it is updated first.
    auto iteration = [&](cudaStream_t q, int i) -> int {
        const int cur = i & 1, prev = cur ^ 1;
        stomp_topk_kernel<<<B, 32, sizeof(float) * R, q>>>(w.tot[prev], w.topk, R, Ro, B, o.state, o.done);
        stomp_rollouts_kernel<<<dim3((R + ro_kg - 1) / ro_kg, B), 128, ro_smem, q>>>(theta, B, T, D, Rn, Ro, ro_kg,
                                                              o.band, w.amp, key0, key1,
                                                              m->dev.lower, m->dev.upper, w.roll[cur], w.roll[prev],
                                                              w.noise, w.sc[cur], w.sc[prev], w.opt_sc, w.topk,
                                                              w.skip, o.state, o.done);
        PS_TRY_CUDA(cudaGetLastError());
        if (int rc = traj_cost_launch(m, scene, w.roll[cur], (Rn + Ro) * B, T, &cp, w.sc[cur], nullptr, nullptr,
                                      w.skip, q))
            return rc;
        stomp_row_totals_kernel<<<dim3(R, B), tot_threads, tot_smem, q>>>(w.roll[cur], w.sc[cur], w.ctrl, w.tot[cur],
                                                                         B, T, D, P->control_cost_weight, P->delta_t,
                                                                         o.state, o.done);
        stomp_weights_kernel<<<w_grid, 256, 0, q>>>(w.sc[cur], w.ctrl, w.noise, w.delta, B, T, D, R,
                                                    P->exponentiated_cost_sensitivity, o.state, o.done);
        stomp_project_kernel<<<B * D, 64, pj_smem, q>>>(theta, w.delta, o.band, w.colscale, B, T, D, o.state, o.done);
        PS_TRY_CUDA(cudaGetLastError());
        if (int rc = traj_cost_launch(m, scene, theta, B, T, &cp, w.opt_sc, nullptr, nullptr, o.done, q)) return rc;
        if (int rc = opt_validity(m, scene, theta, B, T, D, P->collision_margin, P->check_self,
                                  P->collision_check_step, o, q))
            return rc;
        stomp_bookkeep_kernel<<<B, bk_threads, bk_smem, q>>>(theta, w.opt_sc, o.evalid, o.hit, T, D, cp_total,
                                                             P->num_iterations, P->convergence_eps, P->time_limit_ms,
                                                             o.t0, o.state, o.done, best, o.n_done);
        PS_TRY_CUDA(cudaGetLastError());
        return PS_OK;
    };
    if (int rc = opt_run_chunks(iteration, P->num_iterations + 1, B, o.n_done, s)) return rc;
    opt_finalize_kernel<<<B, 128, 0, s>>>(theta, B, T, D, o.state, best, solved, iterations, best_cost);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}
