// ref_harness.cu -- launches PrismPlan's own CUDA kernels on given inputs.
//
// TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile into
// oracle/_ref/libref_oracle.so from the reference sources where they lie
// (the include path points into the read-only reference checkout); no
// reference source is copied into this repository. The GPU parity tests and
// bench.py's plain-path baseline load it to obtain the reference's outputs and
// timings on exactly the inputs the product sees.
//
// Reference entry points exercised (paths inside code/gpu_planning/cpp/src/):
//   pRRTC::check_collision_scene + check_collision_scene_kernel (planning/pRRTC.cu:2337-2423)
//   ppln::search::evaluate_edges_batch                           (planning/edge_eval.cuh:64-165)
//   CHOMP chomp_state_cost_kernel / chomp_obs_grad_kernel        (planning/chomp.cu:83-188)
//   STOMP stomp_state_cost_kernel                                (planning/stomp.cu:206-245)
//   CHOMP::solve_runtime_scene with CHOMPBuffers                 (planning/chomp.cu:358-600,
//                                                                 planning/chomp_buffers.cu)
//   STOMP::solve_runtime_scene with STOMPBuffers                 (planning/stomp.cu:565-965,
//                                                                 planning/stomp_buffers.cu)
//   ppln::collision::fk_runtime, transform_sphere_to_local,
//   sphere_single_obb_collision, sphere_obb_clearance            (device functions, through
//                                                                 the small wrapper kernels below)
// The reference's 4-thread-per-block kernels are launched with their own
// launch shapes. evaluate_edges_batch is run with compute_clearance = false
// only: its clearance branch issues __shfl_xor_sync(0xf, ...) from lanes
// outside that mask (scene_collision.cuh:379 reached from a 64-thread block).
#include "src/planning/pRRTC.cu"
#include "src/planning/chomp.cu"
#include "src/planning/chomp_buffers.cu"
#include "src/planning/stomp_buffers.cu"
#include "src/planning/stomp.cu"
#include "src/planning/edge_eval.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <map>
#include <vector>

#include "../include/prism_b200.h"

namespace {

struct RefModel {
    ppln::RobotModelDevice dev;
};

struct RefScene {
    ppln::collision::SceneCollisionData d{};
    std::vector<void*> owned;
};

template <typename T>
T* upload(const T* h, size_t n, std::vector<void*>& owned) {
    if (!h || n == 0) return nullptr;
    T* d = nullptr;
    if (cudaMalloc(&d, n * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    owned.push_back(d);
    return d;
}

template <typename T>
std::vector<T> vec(const T* p, size_t n) {
    return (p && n) ? std::vector<T>(p, p + n) : std::vector<T>();
}

// fk_runtime over one configuration per 4-thread block; writes the world
// sphere centres in descriptor order. Shared layout as the reference kernels
// (sphere_pos [n_spheres][BATCH_SIZE][3], T [BATCH_SIZE*FK_T_SLOTS*16], q).
__global__ void harness_fk_kernel(const float* q_all, int n, ppln::RobotModel model, float* out) {
    int idx = blockIdx.x;
    if (idx >= n) return;
    int tid = threadIdx.x;
    extern __shared__ float smem[];
    float* sphere_pos = smem;
    float* T = sphere_pos + model.n_spheres * BATCH_SIZE * 3;
    float* q = T + BATCH_SIZE * ppln::FK_T_SLOTS * 16;
    if (tid == 0)
        for (int d = 0; d < model.n_dof; ++d) q[d] = q_all[idx * model.n_dof + d];
    __syncthreads();
    ppln::collision::fk_runtime(model, q, sphere_pos, T, tid);
    __syncthreads();
    for (int s = tid; s < model.n_spheres; s += 4)
        for (int c = 0; c < 3; ++c)
            out[((size_t)idx * model.n_spheres + s) * 3 + c] = sphere_pos[s * BATCH_SIZE * 3 + c];
}

// Min over spheres of sphere_obb_clearance (radius + margin), the OBB
// min-clearance no reference kernel reduces (scene_min_clearance_runtime is
// ESDF only, scene_collision.cuh:339-384).
__global__ void harness_obb_clearance_kernel(const float* q_all, int n, ppln::RobotModel model,
                                             ppln::collision::SceneCollisionData scene, float margin,
                                             float* out) {
    int idx = blockIdx.x;
    if (idx >= n) return;
    int tid = threadIdx.x;
    extern __shared__ float smem[];
    float* sphere_pos = smem;
    float* T = sphere_pos + model.n_spheres * BATCH_SIZE * 3;
    float* q = T + BATCH_SIZE * ppln::FK_T_SLOTS * 16;
    __shared__ float part[4];
    if (tid == 0)
        for (int d = 0; d < model.n_dof; ++d) q[d] = q_all[idx * model.n_dof + d];
    __syncthreads();
    ppln::collision::fk_runtime(model, q, sphere_pos, T, tid);
    __syncthreads();
    float m = 1000.0f;
    for (int s = tid; s < model.n_spheres; s += 4) {
        float c = ppln::collision::sphere_obb_clearance(
            scene, sphere_pos[s * BATCH_SIZE * 3 + 0], sphere_pos[s * BATCH_SIZE * 3 + 1],
            sphere_pos[s * BATCH_SIZE * 3 + 2], model.spheres[s].w + margin, s,
            scene.sphere_obb_acm_mask);
        m = fminf(m, c);
    }
    part[tid] = m;
    __syncthreads();
    if (tid == 0) out[idx] = fminf(fminf(part[0], part[1]), fminf(part[2], part[3]));
}

// scene_min_clearance_runtime (scene_collision.cuh:339-384) of one
// configuration per block. The block has 4 threads, one lane group, so the
// function's __shfl_xor_sync(0xf, ...) names every lane that calls it.
__global__ void harness_esdf_clearance_kernel(const float* q_all, int n, ppln::RobotModel model,
                                              ppln::collision::SceneCollisionData scene, float margin,
                                              float* out) {
    int idx = blockIdx.x;
    if (idx >= n) return;
    int tid = threadIdx.x;
    extern __shared__ float smem[];
    float* sphere_pos = smem;
    float* T = sphere_pos + model.n_spheres * BATCH_SIZE * 3;
    float* q = T + BATCH_SIZE * ppln::FK_T_SLOTS * 16;
    if (tid == 0)
        for (int d = 0; d < model.n_dof; ++d) q[d] = q_all[idx * model.n_dof + d];
    __syncthreads();
    ppln::collision::fk_runtime(model, q, sphere_pos, T, tid);
    __syncthreads();
    const float m = ppln::collision::scene_min_clearance_runtime(model, sphere_pos, scene, tid, margin);
    if (tid == 0) out[idx] = m;
}

__global__ void harness_to_local_kernel(const float* pose, const float* pts, int n, float* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lx, ly, lz;
    ppln::collision::transform_sphere_to_local(pose + 8 * i, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2],
                                               lx, ly, lz);
    out[3 * i] = lx;
    out[3 * i + 1] = ly;
    out[3 * i + 2] = lz;
}

__global__ void harness_obb_pair_kernel(const float* dims, const float* pose, const float* sph, int n,
                                        uint8_t* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = ppln::collision::sphere_single_obb_collision(dims + 4 * i, pose + 8 * i, sph[4 * i],
                                                          sph[4 * i + 1], sph[4 * i + 2], sph[4 * i + 3]);
}

int last_cuda(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        fprintf(stderr, "ref_harness %s: %s\n", where, cudaGetErrorString(e));
        return 3;
    }
    return 0;
}

size_t state_smem(const ppln::RobotModel& m) {
    return (size_t)(m.n_spheres * BATCH_SIZE * 3 + BATCH_SIZE * ppln::FK_T_SLOTS * 16 + m.n_dof) *
           sizeof(float);
}

}  // namespace

extern "C" {

void* ref_model_create(const ps_model_desc* d) {
    const int nj = d->n_joints;
    std::vector<float> ft = vec(d->fixed_transforms, (size_t)nj * 16);
    std::vector<int> types = vec(d->joint_types, (size_t)nj);
    std::vector<float> aft = d->approx_fixed_transforms ? vec(d->approx_fixed_transforms, (size_t)nj * 16) : ft;
    std::vector<int> atypes = d->approx_joint_types ? vec(d->approx_joint_types, (size_t)nj) : types;
    RefModel* m = new RefModel();
    m->dev = ppln::RobotModelDevice::create(
        d->n_dof, nj, ft, types, vec(d->spheres, (size_t)d->n_spheres * 4),
        vec(d->sphere_to_joint, (size_t)d->n_spheres), vec(d->self_cc_ranges, (size_t)d->n_self_cc_ranges * 3),
        vec(d->approx_spheres, (size_t)d->n_approx_spheres * 4),
        vec(d->approx_sphere_to_joint, (size_t)d->n_approx_spheres),
        vec(d->approx_self_cc_ranges, (size_t)d->n_approx_self_cc_ranges * 3), aft, atypes,
        vec(d->joint_lower, (size_t)d->n_dof), vec(d->joint_upper, (size_t)d->n_dof), {}, {}, {}, {}, {},
        vec(d->joint_parents, (size_t)(d->joint_parents ? nj : 0)),
        vec(d->joint_id_to_dof, (size_t)(d->joint_id_to_dof ? nj : 0)),
        vec(d->t_memory_idx, (size_t)(d->t_memory_idx ? nj : 0)),
        vec(d->dfs_order, (size_t)(d->dfs_order ? nj : 0)));
    return m;
}

void ref_model_destroy(void* p) {
    RefModel* m = (RefModel*)p;
    if (!m) return;
    m->dev.destroy();
    delete m;
}

void* ref_scene_create(const float* obb_dims, const float* obb_pose, const uint8_t* obb_enable, int n_obbs,
                       const float* vparams, const float* vpose, const uint8_t* venable, const float* vfeat,
                       int n_layers, int max_vox, const uint8_t* acm, int n_acm, const uint8_t* obb_acm,
                       int n_obb_acm, const uint8_t* obb_acm_apx, int n_obb_acm_apx) {
    RefScene* s = new RefScene();
    auto& d = s->d;
    d.n_obbs = n_obbs;
    d.obb_dims = upload(obb_dims, (size_t)n_obbs * 4, s->owned);
    d.obb_pose = upload(obb_pose, (size_t)n_obbs * 8, s->owned);
    std::vector<uint8_t> en(n_obbs, 1);
    d.obb_enable = upload(obb_enable ? obb_enable : en.data(), (size_t)n_obbs, s->owned);
    d.n_voxel_layers = n_layers;
    d.max_voxels_per_layer = max_vox;
    if (n_layers > 0) {
        d.voxel_params = upload(vparams, (size_t)n_layers * 4, s->owned);
        d.voxel_pose = upload(vpose, (size_t)n_layers * 8, s->owned);
        std::vector<uint8_t> ven(n_layers, 1);
        d.voxel_enable = upload(venable ? venable : ven.data(), (size_t)n_layers, s->owned);
        d.voxel_features = upload(vfeat, (size_t)n_layers * max_vox, s->owned);
    }
    d.sphere_acm_mask = upload(acm, (size_t)n_acm, s->owned);
    d.sphere_obb_acm_mask = upload(obb_acm, (size_t)n_obb_acm, s->owned);
    d.sphere_obb_acm_mask_approx = upload(obb_acm_apx, (size_t)n_obb_acm_apx, s->owned);
    return s;
}

void ref_scene_destroy(void* p) {
    RefScene* s = (RefScene*)p;
    if (!s) return;
    for (void* q : s->owned) cudaFree(q);
    delete s;
}

// pRRTC::check_collision_scene: host in, host out, synchronous (its own
// cudaMalloc / copy / launch / sync / free per call). Returns elapsed ms.
int ref_check_configs(void* mp, void* sp, const float* q, int n, float margin, uint8_t* hit, float* ms) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    std::vector<char> res(n);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    pRRTC::check_collision_scene(q, n, s->d, m->dev.model, margin, (bool*)res.data());
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    if (ms) cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (int i = 0; i < n; ++i) hit[i] = res[i] ? 1 : 0;
    return last_cuda("check_configs");
}

int ref_fk_spheres(void* mp, const float* q, int n, float* out) {
    RefModel* m = (RefModel*)mp;
    const auto& mod = m->dev.model;
    std::vector<void*> own;
    float* dq = upload(q, (size_t)n * mod.n_dof, own);
    float* dout = nullptr;
    cudaMalloc(&dout, (size_t)n * mod.n_spheres * 3 * sizeof(float));
    harness_fk_kernel<<<n, 4, state_smem(mod)>>>(dq, n, mod, dout);
    int rc = last_cuda("fk");
    cudaMemcpy(out, dout, (size_t)n * mod.n_spheres * 3 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dout);
    for (void* p : own) cudaFree(p);
    return rc;
}

int ref_obb_min_clearance(void* mp, void* sp, const float* q, int n, float margin, float* out) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    const auto& mod = m->dev.model;
    std::vector<void*> own;
    float* dq = upload(q, (size_t)n * mod.n_dof, own);
    float* dout = nullptr;
    cudaMalloc(&dout, (size_t)n * sizeof(float));
    harness_obb_clearance_kernel<<<n, 4, state_smem(mod)>>>(dq, n, mod, s->d, margin, dout);
    int rc = last_cuda("obb_clearance");
    cudaMemcpy(out, dout, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dout);
    for (void* p : own) cudaFree(p);
    return rc;
}

int ref_esdf_min_clearance(void* mp, void* sp, const float* q, int n, float margin, float* out) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    const auto& mod = m->dev.model;
    std::vector<void*> own;
    float* dq = upload(q, (size_t)n * mod.n_dof, own);
    float* dout = nullptr;
    cudaMalloc(&dout, (size_t)n * sizeof(float));
    harness_esdf_clearance_kernel<<<n, 4, state_smem(mod)>>>(dq, n, mod, s->d, margin, dout);
    int rc = last_cuda("esdf_clearance");
    cudaMemcpy(out, dout, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dout);
    for (void* p : own) cudaFree(p);
    return rc;
}

int ref_transform_to_local(const float* pose, const float* pts, int n, float* out) {
    std::vector<void*> own;
    float* dp = upload(pose, (size_t)n * 8, own);
    float* dx = upload(pts, (size_t)n * 3, own);
    float* dout = nullptr;
    cudaMalloc(&dout, (size_t)n * 3 * sizeof(float));
    harness_to_local_kernel<<<(n + 127) / 128, 128>>>(dp, dx, n, dout);
    int rc = last_cuda("to_local");
    cudaMemcpy(out, dout, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dout);
    for (void* p : own) cudaFree(p);
    return rc;
}

int ref_obb_pairs(const float* dims, const float* pose, const float* sph, int n, uint8_t* out) {
    std::vector<void*> own;
    float* dd = upload(dims, (size_t)n * 4, own);
    float* dp = upload(pose, (size_t)n * 8, own);
    float* ds = upload(sph, (size_t)n * 4, own);
    uint8_t* dout = nullptr;
    cudaMalloc(&dout, (size_t)n);
    harness_obb_pair_kernel<<<(n + 127) / 128, 128>>>(dd, dp, ds, n, dout);
    int rc = last_cuda("obb_pairs");
    cudaMemcpy(out, dout, (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(dout);
    for (void* p : own) cudaFree(p);
    return rc;
}

// evaluate_edges_batch with a fixed granularity per launch: edges are
// bucketed by their sample count G and each bucket is one <<<E_G, 64>>>
// launch (resolution = 0, granularity = G). Host in/out. *ms = summed
// cudaEvent time of the kernel launches (inputs already resident).
int ref_check_edges(void* mp, void* sp, const float* from, const float* to, const int* G, int n,
                    float margin, int check_self, uint8_t* valid, float* cost, float* ms, int reps) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    const auto& mod = m->dev.model;
    const int D = mod.n_dof;
    std::map<int, std::vector<int>> buckets;
    for (int e = 0; e < n; ++e) buckets[G[e]].push_back(e);
    std::vector<float> hf((size_t)n * D), ht((size_t)n * D);
    std::vector<int> order;
    std::vector<std::pair<int, int>> ranges;   // (offset, count) per bucket, granularity
    std::vector<int> gran;
    for (auto& kv : buckets) {
        ranges.push_back({(int)order.size(), (int)kv.second.size()});
        gran.push_back(kv.first);
        for (int e : kv.second) order.push_back(e);
    }
    for (int k = 0; k < n; ++k) {
        std::copy(from + (size_t)order[k] * D, from + (size_t)(order[k] + 1) * D, hf.begin() + (size_t)k * D);
        std::copy(to + (size_t)order[k] * D, to + (size_t)(order[k] + 1) * D, ht.begin() + (size_t)k * D);
    }
    std::vector<void*> own;
    float* df = upload(hf.data(), hf.size(), own);
    float* dt = upload(ht.data(), ht.size(), own);
    uint8_t* dv = nullptr;
    float *dc = nullptr, *dcl = nullptr;
    cudaMalloc(&dv, n);
    cudaMalloc(&dc, (size_t)n * sizeof(float));
    cudaMalloc(&dcl, (size_t)n * sizeof(float));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float total = 0.0f;
    for (int r = 0; r < std::max(1, reps); ++r) {
        cudaEventRecord(a);
        for (size_t k = 0; k < ranges.size(); ++k) {
            ppln::search::EdgeEvalParams p{};
            p.granularity = gran[k];
            p.collision_margin = margin;
            p.check_self = check_self != 0;
            p.compute_clearance = false;
            p.enable_mesh = false;
            p.resolution = 0.0f;
            int off = ranges[k].first, cnt = ranges[k].second;
            ppln::search::evaluate_edges_batch<<<cnt, 64>>>(df + (size_t)off * D, dt + (size_t)off * D, cnt, D,
                                                            s->d, mod, p, dv + off, dc + off, dcl + off);
        }
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        total += t;
    }
    if (ms) *ms = total / std::max(1, reps);
    int rc = last_cuda("edges");
    std::vector<uint8_t> hv(n);
    std::vector<float> hc(n);
    cudaMemcpy(hv.data(), dv, n, cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), dc, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    for (int k = 0; k < n; ++k) {
        valid[order[k]] = hv[k];
        cost[order[k]] = hc[k];
    }
    cudaFree(dv);
    cudaFree(dc);
    cudaFree(dcl);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (void* p : own) cudaFree(p);
    return rc;
}

// CHOMP per-trajectory kernels in the reference's launch shapes, one
// trajectory at a time (theta [B][D][T], the reference's theta[d*T+t] per
// trajectory). state_costs / obs_grad are [B][D][T]. Either output may be NULL.
// *ms = cudaEvent time of all launches over `reps` repetitions (average).
int ref_chomp(void* mp, void* sp, const float* theta, int B, int T, float w, float world_margin,
              float self_margin, float fd_eps, float* state_costs, float* obs_grad, float* ms, int reps) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    const auto& mod = m->dev.model;
    const int D = mod.n_dof;
    const size_t per = (size_t)D * T;
    std::vector<void*> own;
    float* dth = upload(theta, per * B, own);
    float *dsc = nullptr, *dg = nullptr;
    cudaMalloc(&dsc, per * B * sizeof(float));
    cudaMalloc(&dg, per * B * sizeof(float));
    size_t smem = state_smem(mod);
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(CHOMP::chomp_obs_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(CHOMP::chomp_state_cost_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float total = 0.0f;
    for (int r = 0; r < std::max(1, reps); ++r) {
        cudaEventRecord(a);
        for (int bi = 0; bi < B; ++bi) {
            if (state_costs)
                CHOMP::chomp_state_cost_kernel<<<T, 4, smem>>>(dth + per * bi, dsc + per * bi, mod, s->d, D, T, w,
                                                               world_margin, self_margin);
            if (obs_grad)
                CHOMP::chomp_obs_grad_kernel<<<dim3(T, D), 4, smem>>>(dth + per * bi, dg + per * bi, mod, s->d, D, T,
                                                                      w, world_margin, self_margin, fd_eps);
        }
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        total += t;
    }
    if (ms) *ms = total / std::max(1, reps);
    int rc = last_cuda("chomp");
    if (state_costs) cudaMemcpy(state_costs, dsc, per * B * sizeof(float), cudaMemcpyDeviceToHost);
    if (obs_grad) cudaMemcpy(obs_grad, dg, per * B * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dsc);
    cudaFree(dg);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (void* p : own) cudaFree(p);
    return rc;
}

// CHOMP::solve_runtime_scene once per request, with one CHOMPBuffers set
// reused across requests as chomp_plugin.py does. starts / goals [B][D];
// path [B][T][D], solved [B], iters [B], total [B] (final_total_cost) out,
// all host. include_self / check_self are not settings of the reference
// (it always includes both). *ms = host wall time of the B solves.
int ref_chomp_solve(void* mp, void* sp, const float* starts, const float* goals, int B, int T,
                    const ps_chomp_params* P, float* path, uint8_t* solved, int* iters, float* total,
                    double* ms) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    ppln::RobotModel& mod = m->dev.model;
    const int D = mod.n_dof;
    CHOMP_settings st;
    st.num_timesteps = T;
    st.num_iterations = P->num_iterations;
    st.num_iterations_after_valid = P->num_iterations_after_valid;
    st.step_size = P->step_size;
    st.smoothness_weight = P->smoothness_weight;
    st.collision_cost_weight = P->collision_cost_weight;
    st.world_collision_margin = P->world_margin;
    st.self_collision_margin = P->self_margin;
    st.delta_t = P->delta_t;
    st.convergence_eps = P->convergence_eps;
    st.collision_check_step = P->collision_check_step;
    st.collision_margin = P->collision_margin;
    st.time_limit_ms = P->time_limit_ms;
    CHOMPBuffers bufs = CHOMPBuffers::create(D, T);
    const auto t0 = std::chrono::steady_clock::now();
    for (int b = 0; b < B; ++b) {
        std::vector<float> start(starts + (size_t)b * D, starts + (size_t)(b + 1) * D);
        std::vector<std::vector<float>> gl(1, std::vector<float>(goals + (size_t)b * D, goals + (size_t)(b + 1) * D));
        CHOMPResult r = CHOMP::solve_runtime_scene(start, gl, s->d, st, mod, &bufs);
        for (int t = 0; t < T && t < (int)r.path.size(); ++t)
            for (int d = 0; d < D; ++d) path[((size_t)b * T + t) * D + d] = r.path[t][d];
        solved[b] = r.solved ? 1 : 0;
        iters[b] = r.iterations_run;
        total[b] = r.final_total_cost;
    }
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const int rc = last_cuda("chomp_solve");
    bufs.destroy();
    return rc;
}

// STOMP::solve_runtime_scene once per request, with one STOMPBuffers set
// reused across requests as stomp_plugin.py does. Same outputs as
// ref_chomp_solve. The seed is the reference's own (its RNG init is fixed).
int ref_stomp_solve(void* mp, void* sp, const float* starts, const float* goals, int B, int T,
                    const ps_stomp_params* P, float* path, uint8_t* solved, int* iters, float* total,
                    double* ms) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    ppln::RobotModel& mod = m->dev.model;
    const int D = mod.n_dof;
    STOMP_settings st;
    st.num_timesteps = T;
    st.num_iterations = P->num_iterations;
    st.num_iterations_after_valid = P->num_iterations_after_valid;
    st.num_rollouts_new = P->num_rollouts_new;
    st.num_rollouts_old = P->num_rollouts_old;
    st.delta_t = P->delta_t;
    st.control_cost_weight = P->control_cost_weight;
    st.collision_cost_weight = P->collision_cost_weight;
    st.exponentiated_cost_sensitivity = P->exponentiated_cost_sensitivity;
    st.world_collision_margin = P->world_margin;
    st.self_collision_margin = P->self_margin;
    st.convergence_eps = P->convergence_eps;
    st.noise_scale = P->noise_scale;
    st.collision_check_step = P->collision_check_step;
    st.collision_margin = P->collision_margin;
    st.time_limit_ms = P->time_limit_ms;
    STOMPBuffers bufs = STOMPBuffers::create(D, T, st.num_rollouts_new, st.num_rollouts_old, 1);
    const auto t0 = std::chrono::steady_clock::now();
    for (int b = 0; b < B; ++b) {
        std::vector<float> start(starts + (size_t)b * D, starts + (size_t)(b + 1) * D);
        std::vector<std::vector<float>> gl(1, std::vector<float>(goals + (size_t)b * D, goals + (size_t)(b + 1) * D));
        STOMPResult r = STOMP::solve_runtime_scene(start, gl, s->d, st, mod, &bufs);
        for (int t = 0; t < T && t < (int)r.path.size(); ++t)
            for (int d = 0; d < D; ++d) path[((size_t)b * T + t) * D + d] = r.path[t][d];
        solved[b] = r.solved ? 1 : 0;
        iters[b] = r.iterations_run;
        total[b] = r.final_total_cost;
    }
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const int rc = last_cuda("stomp_solve");
    bufs.destroy();
    return rc;
}

// STOMP state cost over n_rows rollouts [n_rows][D][T] in one
// <<<n_rows*T, 4>>> launch (stomp.cu:820). out [n_rows][D][T].
int ref_stomp_state_cost(void* mp, void* sp, const float* rollouts, int n_rows, int T, float w,
                         float world_margin, float self_margin, float* out, float* ms, int reps) {
    RefModel* m = (RefModel*)mp;
    RefScene* s = (RefScene*)sp;
    const auto& mod = m->dev.model;
    const int D = mod.n_dof;
    const size_t tot = (size_t)n_rows * D * T;
    std::vector<void*> own;
    float* dr = upload(rollouts, tot, own);
    float* dout = nullptr;
    cudaMalloc(&dout, tot * sizeof(float));
    size_t smem = state_smem(mod);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(STOMP::stomp_state_cost_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float total = 0.0f;
    for (int r = 0; r < std::max(1, reps); ++r) {
        cudaEventRecord(a);
        STOMP::stomp_state_cost_kernel<<<n_rows * T, 4, smem>>>(dr, dout, mod, s->d, D, T, n_rows, w, world_margin,
                                                                self_margin);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        total += t;
    }
    if (ms) *ms = total / std::max(1, reps);
    int rc = last_cuda("stomp");
    cudaMemcpy(out, dout, tot * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dout);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    for (void* p : own) cudaFree(p);
    return rc;
}

}  // extern "C"
