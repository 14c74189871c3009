// ps_chomp.cu -- batched CHOMP optimiser loop on the device.
//
// The reference runs one CHOMP request at a time through a host state machine
// (CHOMP::solve_runtime_scene, chomp.cu:358-555): per iteration a
// finite-difference obstacle gradient (2*D FK per waypoint), a covariant step
// theta -= step_size * A^-1 (obs_grad + lambda R theta) with dense T x T
// matrices (chomp_update_kernel, chomp.cu:245-294), a cost refresh, a
// validity check that densifies every segment (chomp_validity_kernel,
// chomp.cu:296-349) and host bookkeeping of the best valid trajectory,
// polishing and convergence, with several host round trips.
//
// Here B requests advance together:
//   * the obstacle gradient is the exact adjoint of the summed hinge
//     (waypoint_cost_kernel), one pass for cost and gradient;
//   * R theta is the 5-tap stencil pair and A^-1 = (R + 1e-8 I)^-1 is applied
//     as a banded Cholesky solve (bandwidth 4) in FP64, factored once per call
//     on the device;
//   * validity checks every segment with the persistent edge kernel (samples
//     j / n_sub, n_sub = ceil(max segment length / collision_check_step)) and
//     every waypoint with the configuration kernel, both with the self check;
//   * the bookkeeping (best valid snapshot, polish budget, two-step convergence
//     streak, iteration count) runs per request on the device, and a finished
//     request is skipped by every later kernel.
// The host loop only launches; it reads one counter every few iterations to
// stop once every request has finished.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "ps_costwarp.cuh"

namespace ps {
namespace {

constexpr int kChompMaxT = 1024;   // one block of T threads per (request, DoF)
constexpr int kBand = 4;           // bandwidth of R (5-point stencil pair)

struct ChompState {
    float best_total, prev_total, last_total, pad0;
    int best_valid, streak, polish_left, iters, step, pad1[3];
};

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// R (central T x T block of dt A^T A over the 6-padded 5-point acceleration
// stencil, chomp_precompute.cpp:20-37) + 1e-8 I, factored as L L^T with L
// lower-banded: L[i * 5 + k] = L(i, i - k) for k = 1..4 and L[i * 5] =
// 1 / L(i, i). FP64, one thread.
__global__ void chomp_band_kernel(int T, float dt_f, double* __restrict__ L) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double dt = dt_f, inv_dt2 = 1.0 / (dt * dt);
    const double coeff[7] = {0.0, -1.0 / 12.0, 16.0 / 12.0, -30.0 / 12.0, 16.0 / 12.0, -1.0 / 12.0, 0.0};
    const int pad = 6, Np = T + 12;
    auto A = [&](int r, int c) -> double {   // padded stencil matrix entry
        const int j = c - r;
        return (j >= -3 && j <= 3) ? inv_dt2 * coeff[j + 3] : 0.0;
    };
    auto R = [&](int i, int j) -> double {   // central block entry
        const int ci = i + pad, cj = j + pad;
        double s = 0.0;
        for (int r = max(max(ci, cj) - 3, 0); r <= min(min(ci, cj) + 3, Np - 1); ++r) s += A(r, ci) * A(r, cj);
        return dt * s + (i == j ? 1.0e-8 : 0.0);
    };
    for (int i = 0; i < T; ++i) {
        for (int j = max(0, i - kBand); j <= i; ++j) {
            double s = R(i, j);
            for (int k = max(0, i - kBand); k < j; ++k) s -= L[i * 5 + (i - k)] * L[j * 5 + (j - k)];
            if (i == j) L[i * 5] = 1.0 / sqrt(s > 0.0 ? s : 1.0e-300);
            else L[i * 5 + (i - j)] = s * L[j * 5];
        }
    }
}

__global__ void chomp_init_kernel(ChompState* __restrict__ st, uint8_t* __restrict__ done, int B,
                                  int polish, int* __restrict__ n_done, unsigned long long* __restrict__ t0) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b == 0) {
        *n_done = 0;
        *t0 = now_ns();
    }
    if (b >= B) return;
    ChompState s;
    s.best_total = INFINITY;
    s.prev_total = INFINITY;
    s.last_total = 0.0f;
    s.pad0 = 0.0f;
    s.best_valid = 0;
    s.streak = 0;
    s.polish_left = polish;
    s.iters = 0;
    s.step = 0;
    st[b] = s;
    done[b] = 0;
}

// One block per request: its segments (theta_t -> theta_t+1) as edges with
// n_sub samples each; 0 samples once the request has finished or when one of
// its waypoints already collides (wp_hit, from the configuration check of the
// same iterate), since the trajectory is then invalid whatever its segments.
__global__ void chomp_segments_kernel(const float* __restrict__ theta, int T, int D, float check_step,
                                      const uint8_t* __restrict__ done, const uint8_t* __restrict__ wp_hit,
                                      float* __restrict__ from, float* __restrict__ to, int* __restrict__ G) {
    __shared__ float red[256];
    const int b = blockIdx.x;
    const float* th = theta + (size_t)b * T * D;
    bool any_hit = false;
    for (int t = threadIdx.x; t < T; t += blockDim.x) any_hit |= wp_hit[(size_t)b * T + t] != 0;
    any_hit = __syncthreads_or(any_hit) != 0;
    float mx = 0.0f;
    for (int t = threadIdx.x; t < T - 1; t += blockDim.x) {
        float d2 = 0.0f;   // in order, without contraction, as the host loop of chomp.cu:462-469
        for (int d = 0; d < D; ++d) {
            const float df = __fsub_rn(th[(t + 1) * D + d], th[t * D + d]);
            d2 = __fadd_rn(d2, __fmul_rn(df, df));
        }
        mx = fmaxf(mx, __fsqrt_rn(d2));
    }
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    const float max_seg = red[0];
    int n_sub = 1;   // chomp.cu:471-474; capped so that the cast stays defined
    if (check_step > 0.0f && max_seg > check_step) n_sub = (int)fminf(ceilf(__fdiv_rn(max_seg, check_step)), 1048576.0f);
    const int g = (done[b] || any_hit) ? 0 : n_sub;
    const size_t e0 = (size_t)b * (T - 1);
    for (int i = threadIdx.x; i < (T - 1) * D; i += blockDim.x) {
        from[e0 * D + i] = th[i];
        to[e0 * D + i] = th[D + i];
    }
    for (int t = threadIdx.x; t < T - 1; t += blockDim.x) G[e0 + t] = g;
}

// One block per request: validity (every segment free and every waypoint
// free), the total cost (sum of waypoint costs + lambda theta^T R theta), then
// the reference's bookkeeping (chomp.cu:487-537) for the request's step k
// (k = 0 is the seed evaluation before the loop, k >= 1 follows the k-th
// update), and the copy of theta into best when it improved. The reference
// checks its stop conditions at the top of the next iteration; here they are
// checked at the end of this one, which stops at the same iterate.
__global__ void chomp_bookkeep_kernel(const float* __restrict__ theta, const float* __restrict__ wp_cost,
                                      const uint8_t* __restrict__ seg_valid, const uint8_t* __restrict__ wp_hit,
                                      int T, int D, ps_cost_params P, int n_iter, float conv_eps,
                                      float time_limit_ms, const unsigned long long* __restrict__ t0,
                                      ChompState* __restrict__ state, uint8_t* __restrict__ done,
                                      float* __restrict__ best, int* __restrict__ n_done) {
    extern __shared__ float sh[];   // traj_smooth_block: 2 (T + 12) + blockDim
    __shared__ int s_valid, s_improved;
    const int b = blockIdx.x;
    if (done[b]) return;   // uniform over the block
    const float* th = theta + (size_t)b * T * D;
    if (threadIdx.x == 0) s_valid = 1;
    __syncthreads();
    bool bad = false;
    for (int t = threadIdx.x; t < T - 1; t += blockDim.x) bad |= seg_valid[(size_t)b * (T - 1) + t] == 0;
    for (int t = threadIdx.x; t < T; t += blockDim.x) bad |= wp_hit[(size_t)b * T + t] != 0;
    if (bad) s_valid = 0;   // benign race: every writer stores 0
    const float total = traj_smooth_block([&](int t, int d) { return th[(size_t)t * D + d]; },
                                          [&](int, int, float) {},
                                          [&](int t) { return wp_cost[(size_t)b * T + t]; }, T, D, P, false, sh);
    if (threadIdx.x == 0) {
        ChompState s = state[b];
        const int k = s.step++;   // evaluation of the iterate after k updates
        const bool valid = s_valid != 0;
        bool improved = false, fin = false;
        s.last_total = total;
        if (k == 0) {
            if (valid) {
                s.best_total = total;
                s.best_valid = 1;
                improved = true;
            }
        } else {
            s.iters += 1;
            if (valid && total < s.best_total) {
                s.best_total = total;
                s.best_valid = 1;
                improved = true;
            }
            if (s.best_valid) {
                const float impr = s.prev_total - s.best_total;
                s.streak = (impr >= 0.0f && impr < conv_eps) ? s.streak + 1 : 0;
                s.prev_total = s.best_total;
                s.polish_left -= 1;
                if (s.streak >= 2) fin = true;
            }
        }
        if (k >= n_iter || (s.best_valid && s.polish_left <= 0)) fin = true;
        if (time_limit_ms > 0.0f && (double)(now_ns() - *t0) > (double)time_limit_ms * 1.0e6) fin = true;
        state[b] = s;
        if (fin) {
            done[b] = 1;
            atomicAdd(n_done, 1);
        }
        s_improved = improved;
    }
    __syncthreads();
    if (s_improved)
        for (int i = threadIdx.x; i < T * D; i += blockDim.x) best[(size_t)b * T * D + i] = th[i];
}

// One block per (request, DoF): g = obs_grad + lambda R theta_d with the
// obstacle gradient of the pinned endpoints taken as 0 (chomp.cu:100-104),
// x = (R + 1e-8 I)^-1 g, then theta_t -= step * x_t on the interior
// waypoints, clamped to the limits (chomp.cu:260-293). R theta (two 5-tap
// stencils) and the banded triangular solves (thread 0) run in FP64: the
// solve amplifies an error in g by up to 1 / lambda_min(R) (about 37 at
// T = 64, dt = 0.1), so g is formed without FP32 rounding.
__global__ void chomp_update_kernel(float* __restrict__ theta, const float* __restrict__ grad,
                                    const double* __restrict__ L, const float* __restrict__ lower,
                                    const float* __restrict__ upper, int T, int D, float step, float lambda,
                                    float dt_f, const uint8_t* __restrict__ done) {
    extern __shared__ double shd[];   // th [T + 12], ac [T + 12], x [T], Ls [5 T]
    const int b = blockIdx.x / D, d = blockIdx.x % D;
    if (done[b]) return;
    const int Np = T + 12;
    double* th = shd;
    double* ac = th + Np;
    double* x = ac + Np;
    double* Ls = x + T;   // the factor, staged so that the serial solve reads shared memory
    for (int k = threadIdx.x; k < 5 * T; k += blockDim.x) Ls[k] = L[k];
    float* col = theta + (size_t)b * T * D + d;   // stride D
    for (int k = threadIdx.x; k < Np; k += blockDim.x) {
        const int t = k - 6;
        th[k] = (t >= 0 && t < T) ? (double)col[(size_t)t * D] : 0.0;
    }
    __syncthreads();
    const double c1 = -1.0 / 12.0, c2 = 16.0 / 12.0, c3 = -30.0 / 12.0;
    const double dt = dt_f, inv_dt2 = 1.0 / (dt * dt);
    for (int k = threadIdx.x; k < Np; k += blockDim.x) {
        auto at = [&](int i) { return (i >= 0 && i < Np) ? th[i] : 0.0; };
        ac[k] = (c1 * (at(k - 2) + at(k + 2)) + c2 * (at(k - 1) + at(k + 1)) + c3 * at(k)) * inv_dt2;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const int k = t + 6;
        const double r = (c1 * (ac[k - 2] + ac[k + 2]) + c2 * (ac[k - 1] + ac[k + 1]) + c3 * ac[k]) * inv_dt2 * dt;
        const double og = (t == 0 || t == T - 1) ? 0.0 : (double)grad[((size_t)b * T + t) * D + d];
        x[t] = og + (double)lambda * r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < T; ++i) {   // L y = g
            double s = x[i];
            for (int j = max(0, i - kBand); j < i; ++j) s -= Ls[i * 5 + (i - j)] * x[j];
            x[i] = s * Ls[i * 5];
        }
        for (int i = T - 1; i >= 0; --i) {   // L^T x = y
            double s = x[i];
            for (int j = i + 1; j <= min(T - 1, i + kBand); ++j) s -= Ls[j * 5 + (j - i)] * x[j];
            x[i] = s * Ls[i * 5];
        }
    }
    __syncthreads();
    const float lo = lower[d], hi = upper[d];
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        if (t == 0 || t == T - 1) continue;   // endpoints pinned to start and goal
        const float v = (float)(th[t + 6] - (double)step * x[t]);
        col[(size_t)t * D] = fmaxf(lo, fminf(hi, v));
    }
}

// Requests that never became valid return their last iterate and its cost.
__global__ void chomp_finalize_kernel(const float* __restrict__ theta, int B, int T, int D,
                                      const ChompState* __restrict__ state, float* __restrict__ best,
                                      uint8_t* __restrict__ solved, int* __restrict__ iterations,
                                      float* __restrict__ best_cost) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const ChompState s = state[b];
    if (threadIdx.x == 0) {
        solved[b] = s.best_valid ? 1 : 0;
        iterations[b] = s.iters;
        best_cost[b] = s.best_valid ? s.best_total : s.last_total;
    }
    if (!s.best_valid)
        for (int i = threadIdx.x; i < T * D; i += blockDim.x) best[(size_t)b * T * D + i] = theta[(size_t)b * T * D + i];
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

// Owns the capture stream and graph of one ps_chomp_optimize call.
struct GraphGuard {
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~GraphGuard() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap) cudaStreamDestroy(cap);
    }
};

struct ChompBufs {
    float *grad, *wp, *from, *to, *ecost;
    int *G, *n_done;
    unsigned long long* t0;
    uint8_t *evalid, *hit, *done;
    ChompState* state;
    double* L;
    void* ews;
    size_t ews_bytes;
};

size_t chomp_layout(int B, int T, int D, ChompBufs* out, void* base) {
    const size_t BT = (size_t)std::max(B, 1) * std::max(T, 1), E = (size_t)std::max(B, 1) * std::max(T - 1, 1);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += a256(bytes);
        return o;
    };
    const size_t o_grad = take(4 * BT * D), o_wp = take(4 * BT), o_from = take(4 * E * D), o_to = take(4 * E * D);
    const size_t o_ecost = take(4 * E), o_G = take(4 * E), o_evalid = take(E), o_hit = take(BT);
    const size_t o_done = take((size_t)std::max(B, 1)), o_state = take(sizeof(ChompState) * std::max(B, 1));
    const size_t o_L = take(sizeof(double) * 5 * std::max(T, 1)), o_nd = take(sizeof(int));
    const size_t o_t0 = take(sizeof(unsigned long long));
    const size_t ews_bytes = ps_edges_workspace_bytes((int)E);
    const size_t o_ews = take(ews_bytes);
    if (out) {
        unsigned char* p = reinterpret_cast<unsigned char*>(base);
        out->grad = reinterpret_cast<float*>(p + o_grad);
        out->wp = reinterpret_cast<float*>(p + o_wp);
        out->from = reinterpret_cast<float*>(p + o_from);
        out->to = reinterpret_cast<float*>(p + o_to);
        out->ecost = reinterpret_cast<float*>(p + o_ecost);
        out->G = reinterpret_cast<int*>(p + o_G);
        out->evalid = p + o_evalid;
        out->hit = p + o_hit;
        out->done = p + o_done;
        out->state = reinterpret_cast<ChompState*>(p + o_state);
        out->L = reinterpret_cast<double*>(p + o_L);
        out->n_done = reinterpret_cast<int*>(p + o_nd);
        out->t0 = reinterpret_cast<unsigned long long*>(p + o_t0);
        out->ews = p + o_ews;
        out->ews_bytes = ews_bytes;
    }
    return off;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" size_t ps_chomp_workspace_bytes(const ps_model* m, int B, int T) {
    if (!m || B < 0 || T < 2) return 0;
    return chomp_layout(B, T, m->info.n_dof, nullptr, nullptr);
}

extern "C" int ps_chomp_optimize(const ps_model* m, const ps_scene_view* scene, float* theta, int B, int T,
                                 const ps_chomp_params* P, float* best, uint8_t* solved, int* iterations,
                                 float* best_cost, void* workspace, size_t workspace_bytes, void* stream) {
    PS_NVTX("ps_chomp_optimize");
    clear_error();
    if (!m || !P) return set_error(PS_EINVAL, "model / params is NULL");
    if (B < 0) return set_error(PS_EINVAL, "B < 0");
    if (T < 2 || T > kChompMaxT) return set_error(PS_EINVAL, "T must be in [2, 1024]");
    if (int rc = validate_scene(m, scene)) return rc;
    if (B == 0) return PS_OK;
    if (!theta || !best || !solved || !iterations || !best_cost) return set_error(PS_EINVAL, "NULL output buffer");
    if (P->num_iterations < 0 || P->num_iterations_after_valid < 0)
        return set_error(PS_EINVAL, "negative iteration count");
    if (!(P->delta_t > 0.0f)) return set_error(PS_EINVAL, "delta_t must be > 0");
    if (m->info.n_joints > 255) return set_error(PS_EINVAL, "too many joints");
    const int D = m->info.n_dof;
    if (!workspace || workspace_bytes < ps_chomp_workspace_bytes(m, B, T))
        return set_error(PS_EINVAL, "workspace missing or smaller than ps_chomp_workspace_bytes");
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return set_error(PS_EINVAL, "workspace not 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    ChompBufs w;
    chomp_layout(B, T, D, &w, workspace);

    // obstacle cost and adjoint only: the update adds lambda R theta itself,
    // and the bookkeeping adds lambda theta^T R theta to the total
    ps_cost_params cp{};
    cp.collision_cost_weight = P->collision_cost_weight;
    cp.world_margin = P->world_margin;
    cp.self_margin = P->self_margin;
    cp.include_self = P->include_self;
    cp.smoothness_weight = 0.0f;
    cp.delta_t = P->delta_t;
    cp.layout = PS_LAYOUT_BTD;
    ps_cost_params cp_total = cp;
    cp_total.smoothness_weight = P->smoothness_weight;
    ps_edge_params ep{};
    ep.granularity = 1;
    ep.collision_margin = P->collision_margin;
    ep.check_self = P->check_self;
    const unsigned cfg_flags = P->check_self ? PS_CHECK_SELF : 0u;
    const int E = B * (T - 1);

    cudaStreamCaptureStatus cap_status = cudaStreamCaptureStatusNone;
    PS_TRY_CUDA(cudaStreamIsCapturing(s, &cap_status));
    if (cap_status != cudaStreamCaptureStatusNone)
        return set_error(PS_EINVAL, "ps_chomp_optimize synchronises and cannot be captured");

    chomp_band_kernel<<<1, 1, 0, s>>>(T, P->delta_t, w.L);
    chomp_init_kernel<<<(B + 127) / 128, 128, 0, s>>>(w.state, w.done, B, P->num_iterations_after_valid, w.n_done,
                                                      w.t0);
    PS_TRY_CUDA(cudaGetLastError());
    const int bk_threads = 128;
    const size_t bk_smem = (size_t)(2 * (T + 12) + bk_threads) * sizeof(float);
    if (bk_smem > 48 * 1024)
        PS_TRY_CUDA(cudaFuncSetAttribute(chomp_bookkeep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bk_smem));
    const int up_threads = std::min(T, 256);
    const size_t up_smem = sizeof(double) * (8 * T + 24);
    if (up_smem > 48 * 1024)
        PS_TRY_CUDA(cudaFuncSetAttribute(chomp_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)up_smem));

    // One iteration: evaluate the current iterate (cost, adjoint, validity,
    // bookkeeping), then step every unfinished trajectory. The step index
    // lives in the device state, so every iteration enqueues the same work.
    auto iteration = [&](cudaStream_t q) -> int {
        if (int rc = traj_cost_launch(m, scene, theta, B, T, &cp, w.wp, nullptr, w.grad, w.done, q)) return rc;
        if (int rc = ps_check_configs(m, scene, theta, B * T, P->collision_margin, cfg_flags, w.hit, nullptr, q))
            return rc;
        chomp_segments_kernel<<<B, 256, 0, q>>>(theta, T, D, P->collision_check_step, w.done, w.hit, w.from, w.to,
                                                w.G);
        PS_TRY_CUDA(cudaGetLastError());
        if (int rc = ps_check_edges(m, scene, w.from, w.to, w.G, E, &ep, w.evalid, w.ecost, nullptr, w.ews,
                                    w.ews_bytes, q))
            return rc;
        chomp_bookkeep_kernel<<<B, bk_threads, bk_smem, q>>>(theta, w.wp, w.evalid, w.hit, T, D, cp_total,
                                                             P->num_iterations, P->convergence_eps, P->time_limit_ms,
                                                             w.t0, w.state, w.done, best, w.n_done);
        PS_TRY_CUDA(cudaGetLastError());
        chomp_update_kernel<<<B * D, up_threads, up_smem, q>>>(theta, w.grad, w.L, m->dev.lower, m->dev.upper, T, D,
                                                               P->step_size, P->smoothness_weight, P->delta_t, w.done);
        PS_TRY_CUDA(cudaGetLastError());
        return PS_OK;
    };

    // kChunk iterations are captured once into a graph on a private stream
    // and replayed on the caller's stream; between replays the host reads how
    // many trajectories have finished. Every trajectory finishes by step
    // num_iterations, and finished ones are skipped, so the replays past that
    // point are never needed.
    constexpr int kChunk = 8;
    GraphGuard g;
    PS_TRY_CUDA(cudaStreamCreateWithFlags(&g.cap, cudaStreamNonBlocking));
    PS_TRY_CUDA(cudaStreamBeginCapture(g.cap, cudaStreamCaptureModeThreadLocal));
    int rc = PS_OK;
    for (int i = 0; i < kChunk && rc == PS_OK; ++i) rc = iteration(g.cap);
    const cudaError_t end_err = cudaStreamEndCapture(g.cap, &g.graph);
    if (rc != PS_OK) return rc;
    if (end_err != cudaSuccess) return cuda_error(end_err, "cudaStreamEndCapture (CHOMP iterations)");
    PS_TRY_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    const int n_chunks = (P->num_iterations + 1 + kChunk - 1) / kChunk;
    for (int c = 0; c < n_chunks; ++c) {
        PS_TRY_CUDA(cudaGraphLaunch(g.exec, s));
        if (c + 1 == n_chunks) break;
        int nd = 0;
        PS_TRY_CUDA(cudaMemcpyAsync(&nd, w.n_done, sizeof(int), cudaMemcpyDeviceToHost, s));
        PS_TRY_CUDA(cudaStreamSynchronize(s));
        if (nd >= B) break;
    }
    chomp_finalize_kernel<<<B, 128, 0, s>>>(theta, B, T, D, w.state, best, solved, iterations, best_cost);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}
