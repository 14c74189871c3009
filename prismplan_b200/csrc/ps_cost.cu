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

#include "ps_internal.h"
#include "ps_verdict.cuh"

namespace ps {

namespace {

constexpr int kCostThreads = 64;

struct CostSmem {
    float* pos;    // [NS*3][kCostThreads]
    float* jf;     // [NJ*12][kCostThreads]: axis(3) origin(3) F(3) M(3)
    float* q;      // [kCostThreads*D]
    unsigned char* sph_joint;   // [NS] DFS position of each reordered sphere
};

// Closest-box search for one sphere: min SDF over boxes, its index and
// whether the centre is inside that box.
__device__ __forceinline__ float closest_box(const SceneSmem& sc, float px, float py, float pz,
                                             const uint8_t* acm_row, int& arg, bool& any_box) {
    float mn = 3.0e38f;
    int am = -1;
    for (int o = 0; o < sc.n_obbs; ++o) {
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        if (d < mn) {
            mn = d;
            am = o;
        }
    }
    any_box = am >= 0;
    if (!any_box) {
        arg = -1;
        return 1000.0f;
    }
    if (mn > 0.0f) {
        arg = am;
        return sqrtf(mn);
    }
    // centre inside at least one box: most negative max(q)
    float best = 3.0e38f;
    for (int o = 0; o < sc.n_obbs; ++o) {
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        if (d == 0.0f) {
            float v = fmaxf(qx, fmaxf(qy, qz));
            if (v < best) {
                best = v;
                am = o;
            }
        }
    }
    arg = am;
    return best;
}

// World gradient of the SDF of box o at p.
__device__ __forceinline__ void box_sdf_grad(const ObbPrep& o, float px, float py, float pz, float& gx, float& gy,
                                             float& gz) {
    float lx = fmaf(o.r0.z, pz, fmaf(o.r0.y, py, fmaf(o.r0.x, px, o.r0.w)));
    float ly = fmaf(o.r1.z, pz, fmaf(o.r1.y, py, fmaf(o.r1.x, px, o.r1.w)));
    float lz = fmaf(o.r2.z, pz, fmaf(o.r2.y, py, fmaf(o.r2.x, px, o.r2.w)));
    float qx = fabsf(lx) - o.h.x, qy = fabsf(ly) - o.h.y, qz = fabsf(lz) - o.h.z;
    float cx = fmaxf(qx, 0.0f), cy = fmaxf(qy, 0.0f), cz = fmaxf(qz, 0.0f);
    float ux, uy, uz;
    const float dsq = fmaf(cz, cz, fmaf(cy, cy, cx * cx));
    if (dsq > 0.0f) {
        const float inv = rsqrtf(dsq);
        ux = copysignf(cx * inv, lx);
        uy = copysignf(cy * inv, ly);
        uz = copysignf(cz * inv, lz);
    } else {
        ux = uy = uz = 0.0f;
        if (qx >= qy && qx >= qz) ux = copysignf(1.0f, lx);
        else if (qy >= qz) uy = copysignf(1.0f, ly);
        else uz = copysignf(1.0f, lz);
    }
    gx = o.r0.x * ux + o.r1.x * uy + o.r2.x * uz;
    gy = o.r0.y * ux + o.r1.y * uy + o.r2.y * uz;
    gz = o.r0.z * ux + o.r1.z * uy + o.r2.z * uz;
}

// kGrad: also produce the adjoint. Output layouts follow ps_cost_params.layout.
template <bool kGrad>
__global__ void __launch_bounds__(kCostThreads) waypoint_cost_kernel(
    ModelDev md, ps_scene_view sv, const float* __restrict__ q, int n_rows, int T, ps_cost_params P,
    float* __restrict__ wp_cost, int broadcast_d, float* __restrict__ traj_acc, float* __restrict__ grad,
    unsigned long long* stats) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    if (!stage_model(md, smem, &mbar)) return;
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof, NJ = M.H->n_joints, NS = M.H->n_spheres;
    ObbPrep* obbs = reinterpret_cast<ObbPrep*>(smem + md.bytes_core);
    const int nob = max(sv.n_obbs, 1);
    int* orig = reinterpret_cast<int*>(obbs + nob);
    LayerPrep* layers = reinterpret_cast<LayerPrep*>(orig + ((nob + 3) & ~3));
    CostSmem cs;
    cs.pos = reinterpret_cast<float*>(layers + PS_MAX_LAYERS);
    cs.jf = cs.pos + (size_t)NS * 3 * kCostThreads;
    cs.q = cs.jf + (size_t)NJ * 12 * kCostThreads;
    cs.sph_joint = reinterpret_cast<unsigned char*>(cs.q + kCostThreads * D);
    SceneSmem sc;
    stage_scene(sv, obbs, orig, layers, counters, &bmax, sc);
    for (int p = 0; p < NJ; ++p)
        for (int k = M.J[p].sph_beg + threadIdx.x; k < M.J[p].sph_end; k += blockDim.x) cs.sph_joint[k] = (unsigned char)p;
    __syncthreads();

    const int lane = threadIdx.x;
    const float w = P.collision_cost_weight, wm = P.world_margin, smg = P.self_margin;
    const bool bdt = P.layout == PS_LAYOUT_BDT;
    const long long total = (long long)n_rows * T;
    LaneStats st;
    st.zero();
#define POS(k, c) cs.pos[((k) * 3 + (c)) * kCostThreads + lane]
#define JF(p, c) cs.jf[((p) * 12 + (c)) * kCostThreads + lane]
    for (long long base = (long long)blockIdx.x * kCostThreads; base < total; base += (long long)gridDim.x * kCostThreads) {
        const long long idx = base + lane;
        const bool active = idx < total;
        const int b = active ? (int)(idx / T) : 0;
        const int t = active ? (int)(idx - (long long)b * T) : 0;
        float* qc = cs.q + lane * D;
        if (active)
            for (int d = 0; d < D; ++d) qc[d] = bdt ? q[((size_t)b * D + d) * T + t] : q[((size_t)b * T + t) * D + d];
        if (!active) continue;
        st.v[ST_SAMPLES] += 1;

        Affine s0, s1, Tf;
        affine_identity(s0);
        affine_identity(s1);
        float esdf_sum = 0.0f, obb_sum = 0.0f;
        for (int p = 0; p < NJ; ++p) {
            const JointRec& jr = M.J[p];
            fk_step<false>(jr, p, qc, s0, s1, Tf);
            if (kGrad) {
                const int ax = jr.type >= PS_X_ROT ? jr.type - PS_X_ROT : (jr.type >= PS_X_PRISM ? jr.type : 0);
                JF(p, 0) = Tf.m[0 + ax];
                JF(p, 1) = Tf.m[4 + ax];
                JF(p, 2) = Tf.m[8 + ax];
                JF(p, 3) = Tf.m[3];
                JF(p, 4) = Tf.m[7];
                JF(p, 5) = Tf.m[11];
            }
            float Fx = 0.f, Fy = 0.f, Fz = 0.f, Mx = 0.f, My = 0.f, Mz = 0.f;
            for (int k = jr.sph_beg; k < jr.sph_end; ++k) {
                const float4 sp = M.S[k];
                float px, py, pz;
                sphere_world(Tf, sp.x, sp.y, sp.z, px, py, pz);
                POS(k, 0) = px;
                POS(k, 1) = py;
                POS(k, 2) = pz;
                const int so = M.SO[k];
                float gx = 0.f, gy = 0.f, gz = 0.f;
                if (sc.n_obbs) {
                    const uint8_t* acm =
                        sv.sphere_obb_acm_mask ? sv.sphere_obb_acm_mask + (size_t)so * sv.n_obbs : nullptr;
                    int arg;
                    bool any_box;
                    const float sdf = closest_box(sc, px, py, pz, acm, arg, any_box);
                    st.v[ST_PAIRS] += sc.n_obbs;
                    const float clr = any_box ? sdf - sp.w : 1000.0f;
                    const float hinge = wm - clr;
                    if (hinge > 0.0f) {
                        obb_sum += hinge;
                        if (kGrad) {
                            float ux, uy, uz;
                            box_sdf_grad(sc.obbs[arg], px, py, pz, ux, uy, uz);
                            gx -= w * ux;
                            gy -= w * uy;
                            gz -= w * uz;
                        }
                    }
                }
                if (sc.n_layers) {
                    const uint8_t* eacm =
                        sv.sphere_acm_mask ? sv.sphere_acm_mask + (size_t)so * sv.n_voxel_layers : nullptr;
                    const float clr = sphere_esdf_clearance(sc, sv, px, py, pz, sp.w, eacm, st);
                    esdf_sum += fmaxf(0.0f, wm - clr);
                    // nearest-voxel lookup is piecewise constant: zero gradient
                }
                if (kGrad) {
                    Fx += gx; Fy += gy; Fz += gz;
                    Mx += py * gz - pz * gy;
                    My += pz * gx - px * gz;
                    Mz += px * gy - py * gx;
                }
            }
            if (kGrad) {
                JF(p, 6) = Fx; JF(p, 7) = Fy; JF(p, 8) = Fz;
                JF(p, 9) = Mx; JF(p, 10) = My; JF(p, 11) = Mz;
            }
        }
        // ---- self hinge ----
        float self_h = 0.0f;
        if (P.include_self && M.H->n_self_pairs > 0) {
            float mn = 1000.0f;
            int arg = -1;
            for (int k = 0; k < M.H->n_self_pairs; ++k) {
                const uint32_t pr = __ldg(md.self_pairs + k);
                const int i = pr & 0xffff, j = pr >> 16;
                const float dx = POS(i, 0) - POS(j, 0), dy = POS(i, 1) - POS(j, 1), dz = POS(i, 2) - POS(j, 2);
                const float c = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx))) - (M.S[i].w + M.S[j].w);
                if (c < mn) {
                    mn = c;
                    arg = k;
                }
            }
            st.v[ST_SELF] += M.H->n_self_pairs;
            self_h = fmaxf(0.0f, smg - mn);
            if (kGrad && self_h > 0.0f && arg >= 0) {
                const uint32_t pr = __ldg(md.self_pairs + arg);
                const int i = pr & 0xffff, j = pr >> 16;
                const float dx = POS(i, 0) - POS(j, 0), dy = POS(i, 1) - POS(j, 1), dz = POS(i, 2) - POS(j, 2);
                const float dd = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
                if (dd > 0.0f) {
                    const float s = w / dd;
                    // d cost / d p_i = -w (p_i - p_j)/d ; d cost / d p_j = +w (p_i - p_j)/d
                    const int pi = cs.sph_joint[i], pj = cs.sph_joint[j];
                    const float gix = -s * dx, giy = -s * dy, giz = -s * dz;
                    const float pix = POS(i, 0), piy = POS(i, 1), piz = POS(i, 2);
                    const float pjx = POS(j, 0), pjy = POS(j, 1), pjz = POS(j, 2);
                    JF(pi, 6) += gix; JF(pi, 7) += giy; JF(pi, 8) += giz;
                    JF(pi, 9) += piy * giz - piz * giy;
                    JF(pi, 10) += piz * gix - pix * giz;
                    JF(pi, 11) += pix * giy - piy * gix;
                    JF(pj, 6) -= gix; JF(pj, 7) -= giy; JF(pj, 8) -= giz;
                    JF(pj, 9) -= pjy * giz - pjz * giy;
                    JF(pj, 10) -= pjz * gix - pjx * giz;
                    JF(pj, 11) -= pjx * giy - pjy * gix;
                }
            }
        }
        const float cost = w * (esdf_sum + obb_sum + self_h);
        if (wp_cost) {
            if (broadcast_d)
                for (int d = 0; d < D; ++d) wp_cost[((size_t)b * D + d) * T + t] = cost;
            else
                wp_cost[idx] = cost;
        }
        if (traj_acc) atomicAdd(traj_acc + b, cost);
        if (kGrad) {
            // reverse sweep: subtree sums, then joint gradients
            for (int p = NJ - 1; p >= 1; --p) {
                const JointRec& jr = M.J[p];
                const float Fx = JF(p, 6), Fy = JF(p, 7), Fz = JF(p, 8);
                const float Mx = JF(p, 9), My = JF(p, 10), Mz = JF(p, 11);
                if (jr.dof >= 0 && jr.type != PS_FIXED) {
                    const float ax = JF(p, 0), ay = JF(p, 1), az = JF(p, 2);
                    float gq;
                    if (jr.type >= PS_X_ROT) {
                        const float ox = JF(p, 3), oy = JF(p, 4), oz = JF(p, 5);
                        // M - o x F
                        const float tx = Mx - (oy * Fz - oz * Fy);
                        const float ty = My - (oz * Fx - ox * Fz);
                        const float tz = Mz - (ox * Fy - oy * Fx);
                        gq = ax * tx + ay * ty + az * tz;
                    } else {
                        gq = ax * Fx + ay * Fy + az * Fz;
                    }
                    const size_t gi = bdt ? ((size_t)b * D + jr.dof) * T + t : ((size_t)b * T + t) * D + jr.dof;
                    grad[gi] += gq;   // a DoF may drive several joints
                }
                const int pp = jr.parent_pos;
                JF(pp, 6) += Fx; JF(pp, 7) += Fy; JF(pp, 8) += Fz;
                JF(pp, 9) += Mx; JF(pp, 10) += My; JF(pp, 11) += Mz;
            }
        }
    }
#undef POS
#undef JF
    flush_stats(stats, st);
}

// Per trajectory and DoF: smoothness cost lambda*theta^T R theta and its
// gradient 2*lambda*R theta added to grad; traj_cost += smoothness (+ the
// deterministic sum of waypoint costs when they were written).
__global__ void smoothness_kernel(const float* __restrict__ q, int B, int T, int D, ps_cost_params P,
                                  const float* __restrict__ wp_cost, float* __restrict__ traj_cost,
                                  float* __restrict__ grad) {
    extern __shared__ float sh[];   // theta_ext [T+12], a [T+12], red [blockDim]
    const int b = blockIdx.x;
    if (b >= B) return;
    const bool bdt = P.layout == PS_LAYOUT_BDT;
    const int Np = T + 12;
    float* th = sh;
    float* ac = sh + Np;
    float* red = ac + Np;
    const float c1 = -1.0f / 12.0f, c2 = 16.0f / 12.0f, c3 = -30.0f / 12.0f;
    const float dt = P.delta_t, inv_dt2 = 1.0f / (dt * dt);
    float local = 0.0f;
    for (int d = 0; d < D; ++d) {
        for (int k = threadIdx.x; k < Np; k += blockDim.x) {
            const int t = k - 6;
            th[k] = (t >= 0 && t < T) ? (bdt ? q[((size_t)b * D + d) * T + t] : q[((size_t)b * T + t) * D + d]) : 0.0f;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < Np; k += blockDim.x) {
            auto at = [&](int i) { return (i >= 0 && i < Np) ? th[i] : 0.0f; };
            float a = c1 * (at(k - 2) + at(k + 2)) + c2 * (at(k - 1) + at(k + 1)) + c3 * at(k);
            a *= inv_dt2;
            ac[k] = a;
            local += dt * a * a;   // theta^T R theta = dt * |A theta|^2
        }
        __syncthreads();
        if (grad && P.smoothness_weight != 0.0f) {
            for (int t = threadIdx.x; t < T; t += blockDim.x) {
                const int k = t + 6;
                float r = c1 * (ac[k - 2] + ac[k + 2]) + c2 * (ac[k - 1] + ac[k + 1]) + c3 * ac[k];
                r *= inv_dt2 * dt;   // (R theta)_t
                const size_t gi = bdt ? ((size_t)b * D + d) * T + t : ((size_t)b * T + t) * D + d;
                grad[gi] += 2.0f * P.smoothness_weight * r;
            }
        }
        __syncthreads();
    }
    float s = P.smoothness_weight * local;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0 && traj_cost) {
        float tot = red[0];
        if (wp_cost) {
            float ws = 0.0f;
            for (int t = 0; t < T; ++t) ws += wp_cost[(size_t)b * T + t];
            traj_cost[b] = ws + tot;
        } else {
            traj_cost[b] += tot;
        }
    }
}

size_t cost_smem(const ps_model* m, const ps_scene_view* sv) {
    return (size_t)m->dev.bytes_core + scene_smem_bytes(sv) +
           (size_t)m->info.n_spheres * 3 * kCostThreads * 4 + (size_t)m->info.n_joints * 12 * kCostThreads * 4 +
           (size_t)kCostThreads * m->info.n_dof * 4 + (size_t)m->info.n_spheres + 16;
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

extern "C" int ps_traj_cost(const ps_model* m, const ps_scene_view* scene, const float* q, int B, int T,
                            const ps_cost_params* P, float* waypoint_cost, float* traj_cost, float* grad,
                            void* stream) {
    clear_error();
    if (int rc = check_cost_params(m, scene, q, B, T, P)) return rc;
    if (B == 0 || T == 0) return PS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = cost_smem(m, scene);
    const long long total = (long long)B * T;
    const int grid = (int)std::max<long long>(1, std::min<long long>((total + kCostThreads - 1) / kCostThreads, 1 << 20));
    const bool atomic_traj = traj_cost && !waypoint_cost;
    if (atomic_traj) PS_TRY_CUDA(cudaMemsetAsync(traj_cost, 0, sizeof(float) * B, s));
    if (grad) {
        PS_TRY_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * (size_t)total * m->info.n_dof, s));
        PS_TRY_CUDA(cudaFuncSetAttribute(waypoint_cost_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        mark_start(s);
        waypoint_cost_kernel<true><<<grid, kCostThreads, smem, s>>>(m->dev, *scene, q, B, T, *P, waypoint_cost, 0,
                                                                    atomic_traj ? traj_cost : nullptr, grad, g_stats);
        mark_stop(s);
    } else {
        PS_TRY_CUDA(cudaFuncSetAttribute(waypoint_cost_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        mark_start(s);
        waypoint_cost_kernel<false><<<grid, kCostThreads, smem, s>>>(m->dev, *scene, q, B, T, *P, waypoint_cost, 0,
                                                                     atomic_traj ? traj_cost : nullptr, nullptr, g_stats);
        mark_stop(s);
    }
    PS_TRY_CUDA(cudaGetLastError());
    if (traj_cost || (grad && P->smoothness_weight != 0.0f)) {
        const int threads = 128;
        const size_t sm2 = (size_t)(2 * (T + 12) + threads) * sizeof(float);
        smoothness_kernel<<<B, threads, sm2, s>>>(q, B, T, m->info.n_dof, *P, waypoint_cost, traj_cost, grad);
        PS_TRY_CUDA(cudaGetLastError());
    }
    return PS_OK;
}

extern "C" int ps_rollout_costs(const ps_model* m, const ps_scene_view* scene, const float* rollouts, int n_rows,
                                int T, const ps_cost_params* P, int broadcast_d, float* state_cost, void* stream) {
    clear_error();
    if (int rc = check_cost_params(m, scene, rollouts, n_rows, T, P)) return rc;
    if (!state_cost && n_rows > 0 && T > 0) return set_error(PS_EINVAL, "state_cost is NULL");
    if (broadcast_d && P->layout != PS_LAYOUT_BDT) return set_error(PS_EINVAL, "broadcast_d needs PS_LAYOUT_BDT");
    if (n_rows == 0 || T == 0) return PS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = cost_smem(m, scene);
    const long long total = (long long)n_rows * T;
    const int grid = (int)std::max<long long>(1, std::min<long long>((total + kCostThreads - 1) / kCostThreads, 1 << 20));
    PS_TRY_CUDA(cudaFuncSetAttribute(waypoint_cost_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mark_start(s);
    waypoint_cost_kernel<false><<<grid, kCostThreads, smem, s>>>(m->dev, *scene, rollouts, n_rows, T, *P, state_cost,
                                                                 broadcast_d, nullptr, nullptr, g_stats);
    mark_stop(s);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}
