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
#include <cstring>

#include "ps_costwarp.cuh"
#include "ps_optloop.cuh"

namespace ps {
namespace {

// One block per request: the total cost of the current iterate (sum of
// waypoint costs + lambda theta^T R theta, the same traj_smooth_block as
// ps_traj_cost, so the same bits), then the shared bookkeeping.
__global__ void chomp_bookkeep_kernel(const float* __restrict__ theta, const float* __restrict__ wp_cost,
                                      const uint8_t* __restrict__ seg_valid, const uint8_t* __restrict__ wp_hit,
                                      int T, int D, ps_cost_params P, int n_iter, float conv_eps,
                                      float time_limit_ms, const unsigned long long* __restrict__ t0,
                                      OptState* __restrict__ state, uint8_t* __restrict__ done,
                                      float* __restrict__ best, int* __restrict__ n_done) {
    extern __shared__ float sh[];   // traj_smooth_block: 2 (T + 12) + blockDim
    const int b = blockIdx.x;
    if (done[b]) return;   // uniform over the block
    const float* th = theta + (size_t)b * T * D;
    const float total = traj_smooth_block([&](int t, int d) { return th[(size_t)t * D + d]; },
                                          [&](int, int, float) {},
                                          [&](int t) { return wp_cost[(size_t)b * T + t]; }, T, D, P, false, sh);
    opt_bookkeep_block(b, th, total, seg_valid, wp_hit, T, D, n_iter, conv_eps, time_limit_ms, t0, state, done, best,
                       n_done);
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
    if (threadIdx.x == 0) band_solve(Ls, x, T);
    __syncthreads();
    const float lo = lower[d], hi = upper[d];
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        if (t == 0 || t == T - 1) continue;   // endpoints pinned to start and goal
        const float v = (float)(th[t + 6] - (double)step * x[t]);
        col[(size_t)t * D] = fmaxf(lo, fminf(hi, v));
    }
}

struct ChompBufs {
    OptBufs o;
    float *grad, *wp;
};

size_t chomp_layout(int B, int T, int D, ChompBufs* out, void* base) {
    ChompBufs w;
    Carver c{reinterpret_cast<unsigned char*>(base)};
    const size_t BT = (size_t)std::max(B, 1) * std::max(T, 1);
    opt_carve(c, B, T, D, w.o);
    w.grad = c.take<float>(4 * BT * D);
    w.wp = c.take<float>(4 * BT);
    if (out) *out = w;
    return c.off;
}

}  // namespace
}  // namespace ps

using namespace ps;

extern "C" size_t ps_chomp_workspace_bytes(const ps_model* m, int B, int T) {
    if (!m || B < 0 || T < 2 || (long long)B * T >= (1ll << 31)) return 0;
    return chomp_layout(B, T, m->info.n_dof, nullptr, nullptr);
}

extern "C" int ps_chomp_optimize(const ps_model* m, const ps_scene_view* scene, float* theta, int B, int T,
                                 const ps_chomp_params* P, float* best, uint8_t* solved, int* iterations,
                                 float* best_cost, void* workspace, size_t workspace_bytes, void* stream) {
    PS_NVTX("ps_chomp_optimize");
    clear_error();
    if (!m || !P) return set_error(PS_EINVAL, "model / params is NULL");
    if (B < 0) return set_error(PS_EINVAL, "B < 0");
    if (T < 2 || T > kOptMaxT) return set_error(PS_EINVAL, "T must be in [2, 1024]");
    if ((long long)B * T >= (1ll << 31)) return set_error(PS_EINVAL, "B * T exceeds 2^31");
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
    const OptBufs& o = w.o;

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

    opt_band_kernel<<<1, 1, 0, s>>>(T, P->delta_t, o.band);
    opt_init_kernel<<<(B + 127) / 128, 128, 0, s>>>(o.state, o.done, B, P->num_iterations_after_valid, o.n_done, o.t0);
    PS_TRY_CUDA(cudaGetLastError());
    const int bk_threads = 128;
    const size_t bk_smem = (size_t)(2 * (T + 12) + bk_threads) * sizeof(float);
    if (bk_smem > 48 * 1024)
        PS_TRY_CUDA(allow_smem((const void*)chomp_bookkeep_kernel, bk_smem));
    const int up_threads = std::min(T, 256);
    const size_t up_smem = sizeof(double) * (8 * T + 24);
    if (up_smem > 48 * 1024)
        PS_TRY_CUDA(allow_smem((const void*)chomp_update_kernel, up_smem));

    // One iteration: evaluate the current iterate (cost, adjoint, validity,
    // bookkeeping), then step every unfinished trajectory. The step index
    // lives in the device state, so every iteration enqueues the same work.
    auto iteration = [&](cudaStream_t q, int) -> int {
        if (int rc = traj_cost_launch(m, scene, theta, B, T, &cp, w.wp, nullptr, w.grad, o.done, q)) return rc;
        if (int rc = opt_validity(m, scene, theta, B, T, D, P->collision_margin, P->check_self,
                                  P->collision_check_step, o, q))
            return rc;
        chomp_bookkeep_kernel<<<B, bk_threads, bk_smem, q>>>(theta, w.wp, o.evalid, o.hit, T, D, cp_total,
                                                             P->num_iterations, P->convergence_eps, P->time_limit_ms,
                                                             o.t0, o.state, o.done, best, o.n_done);
        PS_TRY_CUDA(cudaGetLastError());
        chomp_update_kernel<<<B * D, up_threads, up_smem, q>>>(theta, w.grad, o.band, m->dev.lower, m->dev.upper, T,
                                                               D, P->step_size, P->smoothness_weight, P->delta_t,
                                                               o.done);
        PS_TRY_CUDA(cudaGetLastError());
        return PS_OK;
    };
    if (int rc = opt_run_chunks(iteration, P->num_iterations + 1, B, o.n_done, s)) return rc;
    opt_finalize_kernel<<<B, 128, 0, s>>>(theta, B, T, D, o.state, best, solved, iterations, best_cost);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}
