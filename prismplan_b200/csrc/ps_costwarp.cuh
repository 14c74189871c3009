// ps_costwarp.cuh -- building blocks of the cost kernels shared by the
// per-call and batched paths: the block tables (sphere -> joint, DoF -> joint,
// box centres), the box SDF gradient, fail-closed outputs and the
// smoothness term. The per-waypoint cost itself is in ps_costlane.cuh.
#pragma once

#include <algorithm>
#include <cstdint>

#include "ps_internal.h"
#include "ps_verdict.cuh"

namespace ps {
namespace {

constexpr unsigned kCostFull = 0xffffffffu;

// Block-wide tables of the cost kernels, placed after the staged scene:
//   sph_joint[NS]  DFS position of each reordered sphere
//   dof_joint[16]  per DoF: the one joint it drives, -1 none, -2 several
//   jlist[32], njs the joints that carry exact spheres
//   obs[n_obbs]    world centre and circumscribed radius of each box
struct CostBlock {
    const unsigned char* sph_joint;
    const signed char* dof_joint;
    const unsigned char* jlist;
    const int* njs;
    const float4* obs;
    float* wbase;    // first warp's scratch
};

// Fills the block tables (every thread calls it; the caller syncs after).
__device__ __forceinline__ CostBlock cost_block_setup(unsigned char* at, const ModelSmem& M, const SceneSmem& sc,
                                                      int n_obbs_alloc) {
    const int NJ = M.H->n_joints, NS = M.H->n_spheres, D = M.H->n_dof;
    CostBlock cb;
    unsigned char* sj = at;
    signed char* dj = reinterpret_cast<signed char*>(sj + ((NS + 15) & ~15));
    unsigned char* jl = reinterpret_cast<unsigned char*>(dj + 16);
    int* njs = reinterpret_cast<int*>(dj + 48);
    float4* obs = reinterpret_cast<float4*>(dj + 64);
    cb.sph_joint = sj;
    cb.dof_joint = dj;
    cb.jlist = jl;
    cb.njs = njs;
    cb.obs = obs;
    if (threadIdx.x == 0) {
        int n = 0;
        for (int p = 0; p < NJ; ++p)
            if (M.J[p].sph_end > M.J[p].sph_beg) jl[n++] = (unsigned char)p;
        *njs = n;
    }
    cb.wbase = reinterpret_cast<float*>(obs + max(n_obbs_alloc, 1));
    for (int p = 0; p < NJ; ++p)
        for (int k = M.J[p].sph_beg + threadIdx.x; k < M.J[p].sph_end; k += blockDim.x) sj[k] = (unsigned char)p;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        int who = -1;
        for (int p = 1; p < NJ; ++p)
            if (M.J[p].dof == d && M.J[p].type != PS_FIXED) who = who == -1 ? p : -2;
        dj[d] = (signed char)who;
    }
    box_spheres(sc, obs);
    return cb;
}

// Fail-closed outputs of a cost kernel whose model staging gave up: NaN
// waypoint costs and gradient rows for the waypoints idx this block owns
// (ranges of per_block waypoints, grid-strided). The row writer gets the
// waypoint index and D (read from the blob header in global memory).
template <class RowNaN>
__device__ __forceinline__ void cost_fail_closed(const ModelDev& md, long long total, int per_block, RowNaN row_nan) {
    const int D = reinterpret_cast<const BlobHeader*>(md.blob)->n_dof;
    for (long long r0 = (long long)blockIdx.x * per_block; r0 < total; r0 += (long long)gridDim.x * per_block)
        for (int i = threadIdx.x; i < per_block; i += blockDim.x)
            if (r0 + i < total) row_nan(r0 + i, D);
}

__device__ __forceinline__ void load_frame(const float* f, Affine& T) {
    const float4* v = reinterpret_cast<const float4*>(f);
    const float4 a = v[0], b = v[1], c = v[2];
    T.m[0] = a.x; T.m[1] = a.y; T.m[2] = a.z; T.m[3] = a.w;
    T.m[4] = b.x; T.m[5] = b.y; T.m[6] = b.z; T.m[7] = b.w;
    T.m[8] = c.x; T.m[9] = c.y; T.m[10] = c.z; T.m[11] = c.w;
}

__device__ __forceinline__ void store_frame(float* f, const Affine& T) {
    float4* v = reinterpret_cast<float4*>(f);
    v[0] = make_float4(T.m[0], T.m[1], T.m[2], T.m[3]);
    v[1] = make_float4(T.m[4], T.m[5], T.m[6], T.m[7]);
    v[2] = make_float4(T.m[8], T.m[9], T.m[10], T.m[11]);
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

// One trajectory per block (blockDim a power of two): smoothness
// lambda * sum_d theta_d^T R theta_d with R = dt A^T A
// (chomp_precompute.cpp:20-37), A the 5-point second difference over the
// trajectory zero-padded by 6 on each side, applied as two 5-tap stencils
// instead of a dense T x T product. When want_grad, 2 lambda (R theta_d)_t is
// added through g_add(t, d, value). Returns, in thread 0, the block sum of
// lambda * smoothness + sum_t wp_at(t); the summation order depends only on
// T, D and blockDim, so every caller with the same inputs gets the same bits.
// sh: (2 * (T + 12) + blockDim) floats.
template <class QAt, class GAdd, class WpAt>
__device__ float traj_smooth_block(QAt q_at, GAdd g_add, WpAt wp_at, int T, int D, const ps_cost_params& P,
                                   bool want_grad, float* sh) {
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
            th[k] = (t >= 0 && t < T) ? q_at(t, d) : 0.0f;
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
        if (want_grad && P.smoothness_weight != 0.0f) {
            for (int t = threadIdx.x; t < T; t += blockDim.x) {
                const int k = t + 6;
                float r = c1 * (ac[k - 2] + ac[k + 2]) + c2 * (ac[k - 1] + ac[k + 1]) + c3 * ac[k];
                r *= inv_dt2 * dt;   // (R theta)_t
                g_add(t, d, 2.0f * P.smoothness_weight * r);
            }
        }
        __syncthreads();
    }
    float wsum = 0.0f;
    for (int t = threadIdx.x; t < T; t += blockDim.x) wsum += wp_at(t);
    red[threadIdx.x] = P.smoothness_weight * local + wsum;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    const float tot = red[0];
    __syncthreads();   // red is reused by the caller's next trajectory
    return tot;
}

}  // namespace
}  // namespace ps
