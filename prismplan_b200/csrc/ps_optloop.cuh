// ps_optloop.cuh -- pieces shared by the batched trajectory optimisers
// (ps_chomp.cu, ps_stomp.cu): per-request loop state and the reference's
// bookkeeping, the banded factor of the smoothness metric, the densified
// validity check of an iterate, and the graph-chunk driver. Each translation
// unit that includes this header gets its own private copy of the kernels.
//
// Both reference solvers (CHOMP::solve_runtime_scene, chomp.cu:358-600;
// STOMP::solve_runtime_scene, stomp.cu:565-965) run the same host state
// machine around their updates: seed evaluation, best valid snapshot, a
// polish budget once valid, a two-iteration convergence streak, an iteration
// cap and a wall-clock limit. Here it runs per request on the device.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>

#include "ps_internal.h"

namespace ps {
namespace {

constexpr int kOptMaxT = 1024;   // longest trajectory of the optimisers
constexpr int kBand = 4;         // bandwidth of R (5-point stencil pair)

struct OptState {
    float best_total, prev_total, last_total, pad0;
    int best_valid, streak, polish_left, iters, step, pad1[3];
};

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// R (central T x T block of dt A^T A over the 6-padded 5-point acceleration
// stencil, chomp_precompute.cpp:20-37, stomp_precompute.cpp:24-42) + 1e-8 I,
// factored as L L^T with L lower-banded: L[i * 5 + k] = L(i, i - k) for
// k = 1..4 and L[i * 5] = 1 / L(i, i). FP64, one thread.
__global__ void opt_band_kernel(int T, float dt_f, double* __restrict__ L) {
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

// The two triangular halves of the banded solve, serial in one thread. The
// last kBand results stay in registers, so a step's chain is its kBand
// multiply-subtracts (j ascending, as the textbook loop takes them) and no
// shared-memory round trip; the factor entries do not depend on the chain
// and load ahead of it.
static_assert(kBand == 4, "the register windows below hold kBand = 4 values");

// x <- L^-1 x
__device__ __forceinline__ void band_forward(const double* Ls, double* x, int T) {
    double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;   // y[i-4], y[i-3], y[i-2], y[i-1]
#pragma unroll 4
    for (int i = 0; i < T; ++i) {
        const double* l = Ls + i * 5;
        double s = x[i];
        if (i >= 4) s -= l[4] * w0;
        if (i >= 3) s -= l[3] * w1;
        if (i >= 2) s -= l[2] * w2;
        if (i >= 1) s -= l[1] * w3;
        const double y = s * l[0];
        x[i] = y;
        w0 = w1;
        w1 = w2;
        w2 = w3;
        w3 = y;
    }
}

// x <- L^-T x
__device__ __forceinline__ void band_backward(const double* Ls, double* x, int T) {
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;   // x[i+1], x[i+2], x[i+3], x[i+4]
#pragma unroll 4
    for (int i = T - 1; i >= 0; --i) {
        double s = x[i];
        if (i + 1 <= T - 1) s -= Ls[(i + 1) * 5 + 1] * v0;
        if (i + 2 <= T - 1) s -= Ls[(i + 2) * 5 + 2] * v1;
        if (i + 3 <= T - 1) s -= Ls[(i + 3) * 5 + 3] * v2;
        if (i + 4 <= T - 1) s -= Ls[(i + 4) * 5 + 4] * v3;
        const double xi = s * Ls[i * 5];
        x[i] = xi;
        v3 = v2;
        v2 = v1;
        v1 = v0;
        v0 = xi;
    }
}

// x <- (L L^T)^-1 x for the banded factor of opt_band_kernel (Ls: 5 T
// doubles, any memory). Serial, one thread.
__device__ __forceinline__ void band_solve(const double* Ls, double* x, int T) {
    band_forward(Ls, x, T);
    band_backward(Ls, x, T);
}

__global__ void opt_init_kernel(OptState* __restrict__ st, uint8_t* __restrict__ done, int B, int polish,
                                int* __restrict__ n_done, unsigned long long* __restrict__ t0) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b == 0) {
        *n_done = 0;
        *t0 = now_ns();
    }
    if (b >= B) return;
    OptState s;
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
// n_sub = ceil(max segment L2 / check_step) as the host loops compute it
// (chomp.cu:459-474, stomp.cu:739-755): FP32, in order, no contraction.
__global__ void opt_segments_kernel(const float* __restrict__ theta, int T, int D, float check_step,
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
        float d2 = 0.0f;
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
    int n_sub = 1;   // capped so that the cast stays defined
    if (check_step > 0.0f && max_seg > check_step)
        n_sub = (int)fminf(ceilf(__fdiv_rn(max_seg, check_step)), 1048576.0f);
    const int g = (done[b] || any_hit) ? 0 : n_sub;
    const size_t e0 = (size_t)b * (T - 1);
    for (int i = threadIdx.x; i < (T - 1) * D; i += blockDim.x) {
        from[e0 * D + i] = th[i];
        to[e0 * D + i] = th[D + i];
    }
    for (int t = threadIdx.x; t < T - 1; t += blockDim.x) G[e0 + t] = g;
}

// Block-level part of the bookkeeping for request b (call from every thread
// of a one-block-per-request kernel; `total` valid in thread 0): validity =
// every segment and every waypoint free; then the reference's state machine
// (chomp.cu:486-555, stomp.cu:764-889) for the request's step k (k = 0 is the
// seed evaluation before the loop, k >= 1 follows the k-th update); theta is
// copied into best when it improved. The reference checks its stop
// conditions at the top of the next iteration; here they are checked at the
// end of this one, which stops at the same iterate.
__device__ void opt_bookkeep_block(int b, const float* __restrict__ th, float total, const uint8_t* __restrict__ seg_valid,
                                   const uint8_t* __restrict__ wp_hit, int T, int D, int n_iter, float conv_eps,
                                   float time_limit_ms, const unsigned long long* __restrict__ t0,
                                   OptState* __restrict__ state, uint8_t* __restrict__ done, float* __restrict__ best,
                                   int* __restrict__ n_done) {
    __shared__ int s_improved;
    bool bad = false;
    for (int t = threadIdx.x; t < T - 1; t += blockDim.x) bad |= seg_valid[(size_t)b * (T - 1) + t] == 0;
    for (int t = threadIdx.x; t < T; t += blockDim.x) bad |= wp_hit[(size_t)b * T + t] != 0;
    const bool valid = __syncthreads_or(bad) == 0;
    if (threadIdx.x == 0) {
        OptState s = state[b];
        const int k = s.step++;
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

// Requests that never became valid return their last iterate and its cost.
__global__ void opt_finalize_kernel(const float* __restrict__ theta, int B, int T, int D,
                                    const OptState* __restrict__ state, float* __restrict__ best,
                                    uint8_t* __restrict__ solved, int* __restrict__ iterations,
                                    float* __restrict__ best_cost) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const OptState s = state[b];
    if (threadIdx.x == 0) {
        solved[b] = s.best_valid ? 1 : 0;
        iterations[b] = s.iters;
        best_cost[b] = s.best_valid ? s.best_total : s.last_total;
    }
    if (!s.best_valid)
        for (int i = threadIdx.x; i < T * D; i += blockDim.x) best[(size_t)b * T * D + i] = theta[(size_t)b * T * D + i];
}

inline size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

// Bump allocator over a caller's workspace (or a dry run for its size).
struct Carver {
    unsigned char* base;
    size_t off = 0;
    template <class P>
    P* take(size_t bytes) {
        P* p = base ? reinterpret_cast<P*>(base + off) : nullptr;
        off += a256(bytes);
        return p;
    }
};

// Loop state, validity scratch and the edge workspace of B requests of T
// waypoints (the part both optimisers share).
struct OptBufs {
    OptState* state;
    uint8_t *done, *evalid, *hit;
    int *G, *n_done;
    unsigned long long* t0;
    float *from, *to, *ecost;
    double* band;   // 5 T, opt_band_kernel
    void* ews;
    size_t ews_bytes;
};

inline void opt_carve(Carver& c, int B, int T, int D, OptBufs& o) {
    const size_t Bq = (size_t)std::max(B, 1), BT = Bq * std::max(T, 1), E = Bq * std::max(T - 1, 1);
    o.state = c.take<OptState>(sizeof(OptState) * Bq);
    o.done = c.take<uint8_t>(Bq);
    o.evalid = c.take<uint8_t>(E);
    o.hit = c.take<uint8_t>(BT);
    o.G = c.take<int>(4 * E);
    o.n_done = c.take<int>(sizeof(int));
    o.t0 = c.take<unsigned long long>(sizeof(unsigned long long));
    o.from = c.take<float>(4 * E * D);
    o.to = c.take<float>(4 * E * D);
    o.ecost = c.take<float>(4 * E);
    o.band = c.take<double>(sizeof(double) * 5 * std::max(T, 1));
    o.ews_bytes = ps_edges_workspace_bytes((int)E);
    o.ews = c.take<unsigned char>(o.ews_bytes);
}

// Densified validity of the B iterates theta [B][T][D]: every waypoint
// (configuration kernel) and every segment sample (persistent edge kernel,
// G = n_sub), self check as asked. Results in o.hit / o.evalid.
inline int opt_validity(const ps_model* m, const ps_scene_view* scene, const float* theta, int B, int T, int D,
                        float collision_margin, int check_self, float check_step, const OptBufs& o, cudaStream_t q) {
    ps_edge_params ep{};
    ep.granularity = 1;
    ep.collision_margin = collision_margin;
    ep.check_self = check_self;
    if (int rc = ps_check_configs(m, scene, theta, B * T, collision_margin, check_self ? PS_CHECK_SELF : 0u, o.hit,
                                  nullptr, q))
        return rc;
    opt_segments_kernel<<<B, 256, 0, q>>>(theta, T, D, check_step, o.done, o.hit, o.from, o.to, o.G);
    PS_TRY_CUDA(cudaGetLastError());
    return ps_check_edges(m, scene, o.from, o.to, o.G, B * (T - 1), &ep, o.evalid, o.ecost, nullptr, o.ews,
                          o.ews_bytes, q);
}

// Owns the capture stream and graph of one optimiser call.
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

// Captures kChunk calls of iteration(stream, i) (i = 0..kChunk-1, the
// position inside the chunk) once into a graph on a private stream, then
// replays it on s until n_evals iterations have run or every request has
// finished (read between replays). Every request finishes by its last
// evaluation and finished ones are skipped, so replays past that point are
// never needed.
template <class Iter>
int opt_run_chunks(Iter&& iteration, int n_evals, int B, const int* n_done_dev, cudaStream_t s) {
    constexpr int kChunk = 8;
    cudaStreamCaptureStatus cap_status = cudaStreamCaptureStatusNone;
    PS_TRY_CUDA(cudaStreamIsCapturing(s, &cap_status));
    if (cap_status != cudaStreamCaptureStatusNone)
        return set_error(PS_EINVAL, "the optimiser synchronises and cannot be captured");
    GraphGuard g;
    PS_TRY_CUDA(cudaStreamCreateWithFlags(&g.cap, cudaStreamNonBlocking));
    PS_TRY_CUDA(cudaStreamBeginCapture(g.cap, cudaStreamCaptureModeThreadLocal));
    int rc = PS_OK;
    for (int i = 0; i < kChunk && rc == PS_OK; ++i) rc = iteration(g.cap, i);
    const cudaError_t end_err = cudaStreamEndCapture(g.cap, &g.graph);
    if (rc != PS_OK) return rc;
    if (end_err != cudaSuccess) return cuda_error(end_err, "cudaStreamEndCapture (optimiser iterations)");
    PS_TRY_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    const int n_chunks = (n_evals + kChunk - 1) / kChunk;
    for (int c = 0; c < n_chunks; ++c) {
        PS_TRY_CUDA(cudaGraphLaunch(g.exec, s));
        if (c + 1 == n_chunks) break;
        int nd = 0;
        PS_TRY_CUDA(cudaMemcpyAsync(&nd, n_done_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
        PS_TRY_CUDA(cudaStreamSynchronize(s));
        if (nd >= B) break;
    }
    return PS_OK;
}

}  // namespace
}  // namespace ps
