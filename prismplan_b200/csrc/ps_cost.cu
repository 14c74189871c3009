// ps_cost.cu -- trajectory cost (summed hinge + self hinge + smoothness) with
// its exact gradient, and STOMP rollout costs.
//
// Forward cost per waypoint (chomp.cu:151-188 / stomp.cu:206-245):
//   w * ( sum_s relu(m - esdf_clr_s) + sum_s relu(m - min_o obb_clr_s,o)
//         + relu(m_self - min_(i,j) (|p_i - p_j| - r_i - r_j)) )
// over the full sphere set (scene_collision.cuh:394-495,
// runtime_kinematics.cuh:295-330). The reference differentiates this with a
// central finite difference, 2*D extra FK+hinge evaluations per waypoint
// (chomp.cu:83-144); here one forward pass also produces the analytic adjoint:
//   * per sphere, d cost / d p_s = -w * grad(SDF of the closest box) when the
//     hinge is active (outside: R^T (sign(l) * max(q,0)) / |max(q,0)|;
//     inside: sign(l_k) R_k for the largest q_k), plus the self-pair term;
//   * per joint the sphere forces are reduced to F = sum g, M = sum p x g,
//     and a reverse sweep over the DFS order accumulates subtrees:
//     dC/dq_k = a_k . (M_k - o_k x F_k) (revolute), a_k . F_k (prismatic),
//     with a_k the joint axis and o_k its origin in the world.
// Joint frames are recomputed in the pass rather than stored across kernels.
// The smoothness term lambda * theta_d^T R theta_d uses R = dt A^T A
// (chomp_precompute.cpp:20-37) applied as two 5-tap stencils on the
// zero-padded trajectory instead of a dense T x T product.
#include <algorithm>

#include "ps_costlane.cuh"

namespace ps {

namespace {

size_t cost_block_smem(const ps_model* m, const ps_scene_view* sv, bool grad) {
    return lane_block_bytes(m, sv, kLaneCostWarps, grad);
}

// A group of kCostSub lanes per waypoint, kCostSlots consecutive waypoints
// per warp (see ps_costlane.cuh). kGrad: also the adjoint; kStats: count
// executed work. Output layouts follow ps_cost_params.layout. skip (may be
// NULL): rows b with skip[b] != 0 need no output and get none; a warp whose
// rows are all skipped does nothing. A waypoint gets the same bits whichever
// rows share its warp.
template <bool kGrad, bool kStats>
__global__ void __launch_bounds__(kLaneCostWarps * 32, 2) waypoint_cost_kernel(
    ModelDev md, ps_scene_view sv, const float* __restrict__ q, int n_rows, int T, ps_cost_params P,
    float* __restrict__ wp_cost, int broadcast_d, float* __restrict__ traj_acc, float* __restrict__ grad,
    unsigned long long* stats, const uint8_t* __restrict__ skip) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    const bool bdt = P.layout == PS_LAYOUT_BDT;
    if (!stage_model(md, smem, &mbar)) {
        const float nan = __int_as_float(0x7fc00000);
        cost_fail_closed(md, (long long)n_rows * T, kLaneCostWarps * kCostSlots, [&](long long idx, int D) {
            const int b = (int)(idx / T), tt = (int)(idx - (long long)b * T);
            if (wp_cost) {
                if (broadcast_d)
                    for (int d = 0; d < D; ++d) wp_cost[((size_t)b * D + d) * T + tt] = nan;
                else
                    wp_cost[idx] = nan;
            }
            if (traj_acc) atomicAdd(traj_acc + b, nan);
            if (kGrad)
                for (int d = 0; d < D; ++d) grad[bdt ? ((size_t)b * D + d) * T + tt : ((size_t)b * T + tt) * D + d] = nan;
        });
        return;
    }
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof, NJ = M.H->n_joints;
    ObbPrep* obbs = reinterpret_cast<ObbPrep*>(smem + md.bytes_core);
    const int nob = max(sv.n_obbs, 1);
    int* orig = reinterpret_cast<int*>(obbs + nob);
    LayerPrep* layers = reinterpret_cast<LayerPrep*>(orig + ((nob + 3) & ~3));
    SceneSmem sc;
    stage_scene(sv, obbs, orig, layers, counters, &bmax, sc);
    const CostBlock cb = cost_block_setup(reinterpret_cast<unsigned char*>(layers + PS_MAX_LAYERS), M, sc, sv.n_obbs);
    __syncthreads();
    box_limits(sc, const_cast<float4*>(cb.obs));
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / kCostSub, u = lane % kCostSub;
    const int NS = M.H->n_spheres;
    const LaneScratch ws = lane_carve(reinterpret_cast<unsigned char*>(cb.wbase) +
                                          (size_t)warp * lane_warp_bytes(NJ, NS, D, sv.n_obbs, kGrad),
                                      NJ, NS, D, kGrad);
    const long long total = (long long)n_rows * T;
    LaneStats st;
    st.zero();
    for (long long base = ((long long)blockIdx.x * kLaneCostWarps + warp) * kCostSlots; base < total;
         base += (long long)gridDim.x * kLaneCostWarps * kCostSlots) {
        const long long idx = base + slot;
        const long long ic = idx < total ? idx : total - 1;   // past the end: repeat the last waypoint
        const int b = (int)(ic / T), tt = (int)(ic - (long long)b * T);
        const bool live = idx < total && !(skip && skip[b]);
        if (!__any_sync(kCostFull, live)) continue;   // uniform
        for (int d = u; d < D; d += kCostSub)
            lane_put_q(ws, slot, d, bdt ? q[((size_t)b * D + d) * T + tt] : q[((size_t)b * T + tt) * D + d]);
        __syncwarp();
        LaneStats ls;
        ls.zero();
        const float cost = lane_cost<kGrad, kStats>(M, md, sc, sv, P, cb, ws, ls);
        if (!live) continue;
        if (kStats) {
            if (u == 0) ls.v[ST_SAMPLES] += 1;
            for (int k = 0; k < ST_COUNT; ++k) st.v[k] += ls.v[k];
        }
        if (u == 0) {
            if (wp_cost) {
                if (broadcast_d)
                    for (int d = 0; d < D; ++d) wp_cost[((size_t)b * D + d) * T + tt] = cost;
                else
                    wp_cost[idx] = cost;
            }
            if (traj_acc) atomicAdd(traj_acc + b, cost);
        }
        if (kGrad)
            lane_write_grad(M, cb, ws, bdt ? grad + ((size_t)b * D) * T + tt : grad + ((size_t)b * T + tt) * D,
                            bdt ? T : 1);
    }
    if (kStats) flush_stats(stats, st);
}

// Per trajectory: smoothness cost and its gradient added to grad (see
// traj_smooth_block); traj_cost = sum of waypoint costs + smoothness when the
// waypoint costs were written, else traj_cost += smoothness.
__global__ void smoothness_kernel(const float* __restrict__ q, int B, int T, int D, ps_cost_params P,
                                  const float* __restrict__ wp_cost, float* __restrict__ traj_cost,
                                  float* __restrict__ grad, const uint8_t* __restrict__ skip) {
    extern __shared__ float sh[];
    const int b = blockIdx.x;
    if (b >= B || (skip && skip[b])) return;
    const bool bdt = P.layout == PS_LAYOUT_BDT;
    auto idx = [&](int t, int d) { return bdt ? ((size_t)b * D + d) * T + t : ((size_t)b * T + t) * D + d; };
    const float tot = traj_smooth_block(
        [&](int t, int d) { return q[idx(t, d)]; }, [&](int t, int d, float v) { grad[idx(t, d)] += v; },
        [&](int t) { return wp_cost ? wp_cost[(size_t)b * T + t] : 0.0f; }, T, D, P, grad != nullptr, sh);
    if (threadIdx.x == 0 && traj_cost) {
        if (wp_cost) traj_cost[b] = tot;
        else traj_cost[b] += tot;
    }
}

// Grid of a persistent-style launch: every block resident at once, capped by
// the waypoint count. Returns -1 (error set) if a block does not fit.
template <class K>
int cost_grid(K kernel, size_t smem, long long total) {
    if (allow_smem((const void*)kernel, smem) != cudaSuccess) {
        cudaGetLastError();
        return set_error(PS_EINVAL, "cost kernel shared memory exceeds the device limit"), -1;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kLaneCostWarps * 32, smem);
    if (per_sm < 1) return set_error(PS_EINVAL, "cost kernel does not fit on an SM with this model/scene"), -1;
    const long long need = (total + kLaneCostWarps * kCostSlots - 1) / (kLaneCostWarps * kCostSlots);
    return (int)std::max<long long>(1, std::min<long long>(need, (long long)per_sm * sm_count()));
}

int check_cost_params(const ps_model* m, const ps_scene_view* scene, const float* q, int rows, int T,
                      const ps_cost_params* P) {
    if (!m) return set_error(PS_EINVAL, "model is NULL");
    if (!P) return set_error(PS_EINVAL, "params is NULL");
    if (rows < 0 || T < 0) return set_error(PS_EINVAL, "negative size");
    if (rows > 0 && T > 0 && !q) return set_error(PS_EINVAL, "q is NULL");
    if (P->layout != PS_LAYOUT_BTD && P->layout != PS_LAYOUT_BDT) return set_error(PS_EINVAL, "bad layout");
    if (m->info.n_joints > 255) return set_error(PS_EINVAL, "too many joints");
    return validate_scene(m, scene);
}

}  // namespace
}  // namespace ps

using namespace ps;

int ps::traj_cost_launch(const ps_model* m, const ps_scene_view* scene, const float* q, int B, int T,
                         const ps_cost_params* P, float* waypoint_cost, float* traj_cost, float* grad,
                         const uint8_t* skip, cudaStream_t s) {
    if (int rc = check_cost_params(m, scene, q, B, T, P)) return rc;
    if (B == 0 || T == 0) return PS_OK;
    if (T > PS_MAX_TRAJ_LEN && (traj_cost || (grad && P->smoothness_weight != 0.0f)))
        return set_error(PS_EINVAL, "T exceeds PS_MAX_TRAJ_LEN for the smoothness term");
    const long long total = (long long)B * T;
    const bool atomic_traj = traj_cost && !waypoint_cost;
    if (atomic_traj) PS_TRY_CUDA(cudaMemsetAsync(traj_cost, 0, sizeof(float) * B, s));
    if (grad) {
        const size_t smem = cost_block_smem(m, scene, true);
        auto k = g_stats ? waypoint_cost_kernel<true, true> : waypoint_cost_kernel<true, false>;
        const int grid = cost_grid(k, smem, total);
        if (grid < 0) return PS_EINVAL;
        mark_start(s);
        k<<<grid, kLaneCostWarps * 32, smem, s>>>(m->dev, *scene, q, B, T, *P, waypoint_cost, 0,
                                                  atomic_traj ? traj_cost : nullptr, grad, g_stats, skip);
        mark_stop(s);
    } else {
        const size_t smem = cost_block_smem(m, scene, false);
        auto k = g_stats ? waypoint_cost_kernel<false, true> : waypoint_cost_kernel<false, false>;
        const int grid = cost_grid(k, smem, total);
        if (grid < 0) return PS_EINVAL;
        mark_start(s);
        k<<<grid, kLaneCostWarps * 32, smem, s>>>(m->dev, *scene, q, B, T, *P, waypoint_cost, 0,
                                                  atomic_traj ? traj_cost : nullptr, nullptr, g_stats, skip);
        mark_stop(s);
    }
    PS_TRY_CUDA(cudaGetLastError());
    if (traj_cost || (grad && P->smoothness_weight != 0.0f)) {
        const int threads = 128;
        const size_t sm2 = (size_t)(2 * (T + 12) + threads) * sizeof(float);
        if (sm2 > 48 * 1024)
            PS_TRY_CUDA(allow_smem((const void*)smoothness_kernel, sm2));
        smoothness_kernel<<<B, threads, sm2, s>>>(q, B, T, m->info.n_dof, *P, waypoint_cost, traj_cost, grad, skip);
        PS_TRY_CUDA(cudaGetLastError());
    }
    return PS_OK;
}

extern "C" int ps_traj_cost(const ps_model* m, const ps_scene_view* scene, const float* q, int B, int T,
                            const ps_cost_params* P, float* waypoint_cost, float* traj_cost, float* grad,
                            void* stream) {
    PS_NVTX("ps_traj_cost");
    clear_error();
    return traj_cost_launch(m, scene, q, B, T, P, waypoint_cost, traj_cost, grad, nullptr, (cudaStream_t)stream);
}

extern "C" int ps_rollout_costs(const ps_model* m, const ps_scene_view* scene, const float* rollouts, int n_rows,
                                int T, const ps_cost_params* P, int broadcast_d, float* state_cost, void* stream) {
    PS_NVTX("ps_rollout_costs");
    clear_error();
    if (int rc = check_cost_params(m, scene, rollouts, n_rows, T, P)) return rc;
    if (!state_cost && n_rows > 0 && T > 0) return set_error(PS_EINVAL, "state_cost is NULL");
    if (broadcast_d && P->layout != PS_LAYOUT_BDT) return set_error(PS_EINVAL, "broadcast_d needs PS_LAYOUT_BDT");
    if (n_rows == 0 || T == 0) return PS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const long long total = (long long)n_rows * T;
    const size_t smem = cost_block_smem(m, scene, false);
    auto k = g_stats ? waypoint_cost_kernel<false, true> : waypoint_cost_kernel<false, false>;
    const int grid = cost_grid(k, smem, total);
    if (grid < 0) return PS_EINVAL;
    mark_start(s);
    k<<<grid, kLaneCostWarps * 32, smem, s>>>(m->dev, *scene, rollouts, n_rows, T, *P, state_cost, broadcast_d,
                                              nullptr, nullptr, g_stats, nullptr);
    mark_stop(s);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}
