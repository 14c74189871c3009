// ps_costlane.cuh -- per-waypoint summed-hinge cost and its adjoint, shared
// by the trajectory kernels (ps_cost.cu) and the mixed-request batch
// (ps_batch.cu). See ps_cost.cu for the formulation.
#pragma once

#include "ps_internal.h"
#include "ps_verdict.cuh"

namespace ps {
namespace {

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

// Cost (and, with kGrad, the adjoint added into grad_row[d * gstride]) of
// one waypoint whose configuration is qc. pos / jf are this lane's slices of
// the block's shared arrays with lane stride `stride` (SoA by lane).
template <bool kGrad>
__device__ __forceinline__ float waypoint_cost_lane(const ModelSmem& M, const ModelDev& md, const SceneSmem& sc,
                                                const ps_scene_view& sv, const ps_cost_params& P,
                                                const float* qc, float* pos, float* jf,
                                                const unsigned char* sph_joint, int stride, float* grad_row,
                                                int gstride, LaneStats& st) {
    const int NJ = M.H->n_joints;
    const float w = P.collision_cost_weight, wm = P.world_margin, smg = P.self_margin;
#define POS(k, c) pos[((k) * 3 + (c)) * stride]
#define JF(p, c) jf[((p) * 12 + (c)) * stride]
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
                        esdf_sum += hinge;
                        if (kGrad) {
                            gx += w * bgx;
                            gy += w * bgy;
                            gz += w * bgz;
                        }
                    }
                } else {
                    const float clr = sphere_esdf_clearance(sc, sv, px, py, pz, sp.w, eacm, st);
                    esdf_sum += fmaxf(0.0f, wm - clr);
                    // nearest-voxel lookup is piecewise constant: zero gradient
                }
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
                const int pi = sph_joint[i], pj = sph_joint[j];
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
                grad_row[(size_t)jr.dof * gstride] += gq;   // a DoF may drive several joints
            }
            const int pp = jr.parent_pos;
            JF(pp, 6) += Fx; JF(pp, 7) += Fy; JF(pp, 8) += Fz;
            JF(pp, 9) += Mx; JF(pp, 10) += My; JF(pp, 11) += Mz;
        }
    }
#undef POS
#undef JF
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
