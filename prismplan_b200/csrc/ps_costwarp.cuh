// ps_costwarp.cuh -- per-waypoint summed-hinge cost and its adjoint, one
// warp per waypoint. Shared by the trajectory kernels (ps_cost.cu) and the
// mixed-request batch (ps_batch.cu).
//
// Cost of one configuration (chomp.cu:151-188 / stomp.cu:206-245 over
// scene_collision.cuh:394-495 and runtime_kinematics.cuh:295-330):
//   w * ( sum_s relu(m - esdf_clr_s) + sum_s relu(m - min_o obb_clr_s,o)
//         + relu(m_self - min_(i,j) (|p_i - p_j| - r_i - r_j)) ).
// The reference evaluates every sphere against every box and every self pair
// in one thread. Here the 32 lanes of a warp share one waypoint:
//   1. FK (every lane walks the chain; lane p keeps frame p in shared memory);
//   2. per joint, the boxes that can reach any of its spheres within the
//      hinge band are found from the joint's bound sphere (lanes over boxes,
//      one ballot word per 32 boxes): a box farther than R_p + max(m, 0)
//      from the bound centre has sdf > m + r for every sphere of the joint
//      and contributes nothing;
//   3. lanes over spheres: closest candidate box, ESDF, hinge and d/dp;
//   4. self hinge: joint pairs whose bound spheres are within m_self of each
//      other expand their sphere pairs across the lanes; warp argmin;
//   5. adjoint: per joint F = sum g, M = sum p x g (lane per joint), subtree
//      accumulation from the leaves, dC/dq = a . (M - o x F) (revolute) or
//      a . F (prismatic), a/o the joint axis/origin in the world.
// Sums run in a fixed order (lane-strided partials, xor-tree reduction), so a
// waypoint gives the same bits wherever it is evaluated.
#pragma once

#include "ps_internal.h"
#include "ps_verdict.cuh"

namespace ps {
namespace {

constexpr unsigned kCostFull = 0xffffffffu;

// Per-warp scratch in shared memory (floats unless noted).
struct CostWarpScratch {
    float* q;        // [16]
    float* frame;    // [NJ][12]
    float* bnd;      // [NJ][4]: bound centre (world), radius
    float* pos;      // [NS][3]
    float* g;        // [NS][3]   (gradient only)
    float* jfm;      // [NJ][8]: F, M, dC/dq   (gradient only)
    unsigned* mask;  // [NJ][nw]  candidate boxes per joint
};

__host__ __device__ inline int cost_mask_words(int n_obbs) { return (n_obbs + 31) / 32; }

__host__ __device__ inline size_t cost_warp_floats(int NJ, int NS, int n_obbs, bool grad) {
    size_t f = 16 + (size_t)NJ * 12 + (size_t)NJ * 4 + (size_t)NS * 3 + (size_t)NJ * cost_mask_words(n_obbs);
    if (grad) f += (size_t)NS * 3 + (size_t)NJ * 8;
    return (f + 3) & ~size_t(3);   // keep every warp's slice 16-byte aligned
}

__device__ __forceinline__ CostWarpScratch cost_carve(float* base, int NJ, int NS, int n_obbs, bool grad) {
    CostWarpScratch w;
    w.q = base;
    w.frame = w.q + 16;
    w.bnd = w.frame + NJ * 12;
    w.pos = w.bnd + NJ * 4;
    float* p = w.pos + NS * 3;
    if (grad) {
        w.g = p;
        w.jfm = w.g + NS * 3;
        p = w.jfm + NJ * 8;
    } else {
        w.g = nullptr;
        w.jfm = nullptr;
    }
    w.mask = reinterpret_cast<unsigned*>(p);
    return w;
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

// Signed distance to the closest candidate box (ACM row applied): the
// smallest outside distance, or, when the centre lies inside boxes, the most
// negative max(q) among them. Returns false when no candidate is left.
__device__ __forceinline__ bool closest_candidate(const SceneSmem& sc, const unsigned* mask, int nw, float px,
                                                  float py, float pz, const uint8_t* acm_row, float& sdf, int& arg,
                                                  unsigned& tests) {
    float mn = 3.0e38f;
    int am = -1;
    for (int w = 0; w < nw; ++w) {
        unsigned m = mask[w];
        while (m) {
            const int o = w * 32 + __ffs(m) - 1;
            m &= m - 1;
            if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
            float qx, qy, qz;
            const float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
            ++tests;
            if (d < mn) {
                mn = d;
                am = o;
            }
        }
    }
    if (am < 0) return false;
    if (mn > 0.0f) {
        sdf = sqrtf(mn);
        arg = am;
        return true;
    }
    float best = 3.0e38f;
    for (int w = 0; w < nw; ++w) {
        unsigned m = mask[w];
        while (m) {
            const int o = w * 32 + __ffs(m) - 1;
            m &= m - 1;
            if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
            float qx, qy, qz;
            if (fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz) == 0.0f) {
                const float v = fmaxf(qx, fmaxf(qy, qz));
                if (v < best) {
                    best = v;
                    am = o;
                }
            }
        }
    }
    sdf = best;
    arg = am;
    return true;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kCostFull, v, o);
    return v;
}

// Cost (returned on every lane) and, with kGrad, d cost / d q written by
// lanes d < n_dof to grad_row[d * gstride]. The whole warp calls it; the
// configuration is ws.q[0..D).
template <bool kGrad>
__device__ float waypoint_cost_warp(const ModelSmem& M, const ModelDev& md, const SceneSmem& sc,
                                    const ps_scene_view& sv, const ps_cost_params& P,
                                    const unsigned char* sph_joint, const CostWarpScratch& ws, float* grad_row,
                                    int gstride, LaneStats& st) {
    const int lane = threadIdx.x & 31;
    const int D = M.H->n_dof, NJ = M.H->n_joints, NS = M.H->n_spheres;
    const float w = P.collision_cost_weight, wm = P.world_margin, smg = P.self_margin;
    const int nob = sc.n_obbs, nw = cost_mask_words(nob);

    // ---- 1. FK: every lane walks the chain, lane p stores frame p ----
    {
        Affine s0, s1, Tf;
        affine_identity(s0);
        affine_identity(s1);
        for (int p = 0; p < NJ; ++p) {
            fk_step<false>(M.J[p], p, ws.q, s0, s1, Tf);
            if (lane == (p & 31)) {
#pragma unroll
                for (int i = 0; i < 12; ++i) ws.frame[p * 12 + i] = Tf.m[i];
            }
        }
        if (lane == 0) st.v[ST_JOINTS] += NJ;
    }
    __syncwarp();
    // bound sphere of each joint in the world
    for (int p = lane; p < NJ; p += 32) {
        const float4 b = M.J[p].bound;
        Affine T;
#pragma unroll
        for (int i = 0; i < 12; ++i) T.m[i] = ws.frame[p * 12 + i];
        float cx = 0.f, cy = 0.f, cz = 0.f;
        if (b.w >= 0.0f) sphere_world(T, b.x, b.y, b.z, cx, cy, cz);
        ws.bnd[p * 4 + 0] = cx;
        ws.bnd[p * 4 + 1] = cy;
        ws.bnd[p * 4 + 2] = cz;
        ws.bnd[p * 4 + 3] = b.w;
    }
    __syncwarp();

    // ---- 2. candidate boxes per joint (lanes over boxes) ----
    if (nob > 0) {
        const float mpos = fmaxf(wm, 0.0f);
        for (int base = 0; base < nob; base += 32) {
            const int o = base + lane;
            const bool ok = o < nob;
            ObbPrep box;
            if (ok) box = sc.obbs[o];
            for (int p = 0; p < NJ; ++p) {
                const float R = ws.bnd[p * 4 + 3];
                bool keep = false;
                if (R >= 0.0f && ok) {
                    const float cx = ws.bnd[p * 4 + 0], cy = ws.bnd[p * 4 + 1], cz = ws.bnd[p * 4 + 2];
                    // slack for the FP32 rounding of the transforms and the test
                    const float S = fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz)));
                    float thr = R + mpos;
                    thr += 4.0f * (S + thr + sc.Bmax + 1.0f) * PS_GUARD_K;
                    float qx, qy, qz;
                    keep = fast_box_dsq(box, cx, cy, cz, qx, qy, qz) < thr * thr;
                    st.v[ST_CULL] += 1;
                }
                const unsigned bal = __ballot_sync(kCostFull, keep);
                if (lane == 0) ws.mask[p * nw + (base >> 5)] = bal;
            }
        }
        __syncwarp();
    }

    // ---- 3. spheres (lanes over spheres) ----
    float obb_part = 0.0f, esdf_part = 0.0f;
    for (int k = lane; k < NS; k += 32) {
        const int p = sph_joint[k];
        const float4 sp = M.S[k];
        Affine T;
#pragma unroll
        for (int i = 0; i < 12; ++i) T.m[i] = ws.frame[p * 12 + i];
        float px, py, pz;
        sphere_world(T, sp.x, sp.y, sp.z, px, py, pz);
        ws.pos[k * 3 + 0] = px;
        ws.pos[k * 3 + 1] = py;
        ws.pos[k * 3 + 2] = pz;
        st.v[ST_SPHERES] += 1;
        const int so = M.SO[k];
        float gx = 0.f, gy = 0.f, gz = 0.f;
        if (nob > 0) {
            const uint8_t* acm = sv.sphere_obb_acm_mask ? sv.sphere_obb_acm_mask + (size_t)so * sv.n_obbs : nullptr;
            float sdf;
            int arg;
            unsigned tests = 0;
            if (closest_candidate(sc, ws.mask + p * nw, nw, px, py, pz, acm, sdf, arg, tests)) {
                const float hinge = wm - (sdf - sp.w);
                if (hinge > 0.0f) {
                    obb_part += hinge;
                    if (kGrad) {
                        float ux, uy, uz;
                        box_sdf_grad(sc.obbs[arg], px, py, pz, ux, uy, uz);
                        gx -= w * ux;
                        gy -= w * uy;
                        gz -= w * uz;
                    }
                }
            }
            st.v[ST_PAIRS] += tests;
        }
        if (sc.n_layers) {
            const uint8_t* eacm = sv.sphere_acm_mask ? sv.sphere_acm_mask + (size_t)so * sv.n_voxel_layers : nullptr;
            if (sv.esdf_mode == PS_ESDF_TRILINEAR) {
                // min over layers of -d - r; d(cost)/dp = w * grad d of the minimising layer
                float best = 1000.0f, bgx = 0.f, bgy = 0.f, bgz = 0.f;
                for (int l = 0; l < sc.n_layers; ++l) {
                    if (eacm && eacm[l] == 0) continue;
                    float d, dgx, dgy, dgz;
                    st.v[ST_ESDF] += 1;
                    if (!esdf_sample_trilinear_grad(sc.layers[l], sv.voxel_features + (size_t)l * sv.max_voxels_per_layer,
                                                    sv.max_voxels_per_layer, px, py, pz, d, dgx, dgy, dgz))
                        continue;
                    const float c = -d - sp.w;
                    if (c < best) {
                        best = c;
                        bgx = dgx;
                        bgy = dgy;
                        bgz = dgz;
                    }
                }
                const float hinge = wm - best;
                if (hinge > 0.0f) {
                    esdf_part += hinge;
                    if (kGrad) {
                        gx += w * bgx;
                        gy += w * bgy;
                        gz += w * bgz;
                    }
                }
            } else {
                const float clr = sphere_esdf_clearance(sc, sv, px, py, pz, sp.w, eacm, st);
                esdf_part += fmaxf(0.0f, wm - clr);
                // the nearest-voxel lookup is piecewise constant: zero gradient
            }
        }
        if (kGrad) {
            ws.g[k * 3 + 0] = gx;
            ws.g[k * 3 + 1] = gy;
            ws.g[k * 3 + 2] = gz;
        }
    }
    __syncwarp();

    // ---- 4. self hinge: joint-pair prefilter, then sphere pairs ----
    float self_h = 0.0f;
    int self_arg = -1;
    if (P.include_self && md.n_jpairs > 0) {
        float bv = 3.0e38f;
        int bk = 0x7fffffff;
        for (int base = 0; base < md.n_jpairs; base += 32) {
            const int gi = base + lane;
            bool act = false;
            int4 jp = make_int4(0, 0, 0, 0);
            if (gi < md.n_jpairs) {
                jp = __ldg(md.jpairs + gi);
                const float* A = ws.bnd + jp.x * 4;
                const float* B = ws.bnd + jp.y * 4;
                const float dx = A[0] - B[0], dy = A[1] - B[1], dz = A[2] - B[2];
                const float S = fmaxf(fmaxf(fabsf(A[0]), fabsf(A[1])), fmaxf(fabsf(A[2]), fmaxf(fabsf(B[0]),
                                fmaxf(fabsf(B[1]), fabsf(B[2])))));
                float thr = A[3] + B[3] + fmaxf(smg, 0.0f);
                thr += 4.0f * (S + thr + 1.0f) * PS_GUARD_K;
                act = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) < thr * thr;
                st.v[ST_SELF] += 1;
            }
            unsigned todo = __ballot_sync(kCostFull, act);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const int beg = __shfl_sync(kCostFull, jp.z, src), end = __shfl_sync(kCostFull, jp.w, src);
                for (int k = beg + lane; k < end; k += 32) {
                    const uint32_t pr = __ldg(md.gpairs + k);
                    const int i = pr & 0xffff, j = pr >> 16;
                    const float dx = ws.pos[i * 3] - ws.pos[j * 3], dy = ws.pos[i * 3 + 1] - ws.pos[j * 3 + 1],
                                dz = ws.pos[i * 3 + 2] - ws.pos[j * 3 + 2];
                    const float c = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx))) - (M.S[i].w + M.S[j].w);
                    if (c < bv || (c == bv && k < bk)) {
                        bv = c;
                        bk = k;
                    }
                    st.v[ST_SELF] += 1;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(kCostFull, bv, o);
            const int ok = __shfl_xor_sync(kCostFull, bk, o);
            if (ov < bv || (ov == bv && ok < bk)) {
                bv = ov;
                bk = ok;
            }
        }
        self_h = fmaxf(0.0f, smg - bv);
        self_arg = self_h > 0.0f ? bk : -1;
    }
    const float cost = w * (warp_sum(esdf_part) + warp_sum(obb_part) + self_h);
    if (!kGrad) return cost;

    // ---- 5. adjoint ----
    if (self_arg >= 0 && lane == 0) {
        const uint32_t pr = __ldg(md.gpairs + self_arg);
        const int i = pr & 0xffff, j = pr >> 16;
        const float dx = ws.pos[i * 3] - ws.pos[j * 3], dy = ws.pos[i * 3 + 1] - ws.pos[j * 3 + 1],
                    dz = ws.pos[i * 3 + 2] - ws.pos[j * 3 + 2];
        const float dd = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
        if (dd > 0.0f) {
            // d cost / d p_i = -w (p_i - p_j)/d ; d cost / d p_j = +w (p_i - p_j)/d
            const float s = w / dd;
            ws.g[i * 3 + 0] -= s * dx;
            ws.g[i * 3 + 1] -= s * dy;
            ws.g[i * 3 + 2] -= s * dz;
            ws.g[j * 3 + 0] += s * dx;
            ws.g[j * 3 + 1] += s * dy;
            ws.g[j * 3 + 2] += s * dz;
        }
    }
    __syncwarp();
    // per joint: F = sum g, M = sum p x g over its own spheres
    for (int p = lane; p < NJ; p += 32) {
        float Fx = 0.f, Fy = 0.f, Fz = 0.f, Mx = 0.f, My = 0.f, Mz = 0.f;
        for (int k = M.J[p].sph_beg; k < M.J[p].sph_end; ++k) {
            const float gx = ws.g[k * 3], gy = ws.g[k * 3 + 1], gz = ws.g[k * 3 + 2];
            const float px = ws.pos[k * 3], py = ws.pos[k * 3 + 1], pz = ws.pos[k * 3 + 2];
            Fx += gx; Fy += gy; Fz += gz;
            Mx += py * gz - pz * gy;
            My += pz * gx - px * gz;
            Mz += px * gy - py * gx;
        }
        float* f = ws.jfm + p * 8;
        f[0] = Fx; f[1] = Fy; f[2] = Fz; f[3] = Mx; f[4] = My; f[5] = Mz;
    }
    __syncwarp();
    // subtree sums from the leaves (children follow their parent in DFS order);
    // lane c < 6 owns component c
    if (lane < 6)
        for (int p = NJ - 1; p >= 1; --p) ws.jfm[M.J[p].parent_pos * 8 + lane] += ws.jfm[p * 8 + lane];
    __syncwarp();
    for (int p = lane; p < NJ; p += 32) {
        const JointRec& jr = M.J[p];
        float gq = 0.0f;
        if (p >= 1 && jr.dof >= 0 && jr.type != PS_FIXED) {
            const float* f = ws.jfm + p * 8;
            const float* T = ws.frame + p * 12;
            const int ax = jr.type >= PS_X_ROT ? jr.type - PS_X_ROT : (jr.type >= PS_X_PRISM ? jr.type : 0);
            const float axx = T[0 + ax], axy = T[4 + ax], axz = T[8 + ax];
            if (jr.type >= PS_X_ROT) {
                const float ox = T[3], oy = T[7], oz = T[11];
                // M - o x F
                const float tx = f[3] - (oy * f[2] - oz * f[1]);
                const float ty = f[4] - (oz * f[0] - ox * f[2]);
                const float tz = f[5] - (ox * f[1] - oy * f[0]);
                gq = axx * tx + axy * ty + axz * tz;
            } else {
                gq = axx * f[0] + axy * f[1] + axz * f[2];
            }
        }
        ws.jfm[p * 8 + 6] = gq;
    }
    __syncwarp();
    // a DoF may drive several joints: lane d sums its joints in DFS order
    for (int d = lane; d < D; d += 32) {
        float acc = 0.0f;
        for (int p = 1; p < NJ; ++p)
            if (M.J[p].dof == d && M.J[p].type != PS_FIXED) acc += ws.jfm[p * 8 + 6];
        grad_row[(size_t)d * gstride] = acc;
    }
    __syncwarp();
    return cost;
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
