// ps_costlane.cuh -- per-waypoint summed-hinge cost and its adjoint, a group
// of kCostSub lanes per waypoint. Shared by the trajectory kernels
// (ps_cost.cu) and the mixed-request batch (ps_batch.cu).
//
// Cost of one configuration (chomp.cu:151-188 / stomp.cu:206-245 over
// scene_collision.cuh:394-495 and runtime_kinematics.cuh:295-330):
//   w * ( sum_s relu(m - esdf_clr_s) + sum_s relu(m - min_o obb_clr_s,o)
//         + relu(m_self - min_(i,j) (|p_i - p_j| - r_i - r_j)) ).
// A warp holds kCostSlots waypoints, kCostSub lanes each; every loop below is
// uniform over the warp (candidate lists, runs, joint pairs), so lanes do not
// diverge on them:
//   1. FK walk in DFS order with accurate sincosf (each lane of a group
//      repeats it; the group's frames, each joint's world bound centre and,
//      in step 3, each sphere's world centre go to shared memory, SoA by
//      waypoint slot);
//   2. per joint, one warp broad phase: the joint's bound spheres of the
//      warp's waypoints are enclosed by one sphere (centre = lane 16's, radius
//      = a one-instruction warp max), and lanes over boxes keep the boxes
//      within that radius + max(m, 0) (a circumscribed-sphere test first, the
//      box distance second). A box outside it has sdf > m + r for every sphere
//      of the joint at every waypoint of the warp, so it changes no hinge;
//   3. the joint's spheres, split over the group's lanes, up to 4 per box load,
//      against the kept boxes: the closest box by one key per pair (d^2
//      outside, the most negative max(q) inside), then sdf, hinge and, with the
//      gradient, the force g = -w grad(sdf) summed into the joint's
//      F = sum g, M = sum p x g;
//   4. F and M are summed over the group and folded into the joint's
//      ancestors: dC/dq_p += a_p . (M - o_p x F) (revolute) or a_p . F
//      (prismatic), a_p and o_p the joint axis and origin from the frames;
//   5. self hinge, on the world sphere centres that step 3 left in shared
//      memory. It is a minimum, so every test culls against the smallest
//      clearance the group has found so far (the cull level; m_self at the
//      start), and the joint pairs come nearest in DFS order first, so that
//      level drops early. The group's lanes split the joint pairs' bound
//      tests (one ballot gives each pair's OR over the warp's waypoints); a
//      pair that can come below the level expands its runs (sphere i of joint
//      a against consecutive spheres j of joint q), split over the group's
//      lanes; a lane skips its run when i is out of reach of q's bound sphere
//      on its own waypoint. A square root is taken only for pairs that can
//      come below the level; the minimum over the group is taken by (value,
//      pair order), and the argmin pair's force goes to both joints'
//      ancestors.
// Every candidate set is a superset of what the waypoint itself needs, and
// the group size is fixed, so a waypoint gives the same bits whatever other
// waypoints share its warp; the batch relies on that.
#pragma once

#include <algorithm>
#include <climits>
#include <cstdint>

#include "ps_costwarp.cuh"

namespace ps {
namespace {

constexpr int kCostSub = 4;                  // lanes per waypoint
constexpr int kCostSlots = 32 / kCostSub;    // waypoints per warp
constexpr int kLaneCostWarps = 8;            // warps per block of the cost kernels

// Per-warp scratch floats, SoA over the warp's waypoint slots: frames of
// joints 1..NJ-1 (joint 0 is the identity), world bound centres, world
// sphere centres, per-joint gradient (gradient only), the waypoint's
// configuration and each DoF's sine and cosine.
__host__ __device__ inline int lane_cost_floats(int NJ, int NS, int D, bool grad) {
    return kCostSlots * (12 * (NJ - 1) + 3 * NJ + 3 * NS + (grad ? NJ : 0) + 3 * D);
}
__host__ __device__ inline size_t lane_warp_bytes(int NJ, int NS, int D, int n_obbs, bool grad) {
    return (size_t)lane_cost_floats(NJ, NS, D, grad) * 4 +
           ((((size_t)(n_obbs > 0 ? n_obbs : 1)) * 2 + 15) & ~size_t(15));
}

struct LaneScratch {
    float* fr;        // [(NJ-1)*12][slots]
    float* bc;        // [NJ*3][slots]
    float* pos;       // [NS*3][slots]
    float* dq;        // [NJ][slots] (gradient only)
    float* q;         // [D][slots]
    float* sc;        // [2*D][slots]: sin, cos of each DoF (accurate sincosf)
    uint16_t* cand;   // [n_obbs]: boxes kept by the current joint's broad phase (warp-uniform)
};

__device__ __forceinline__ LaneScratch lane_carve(unsigned char* base, int NJ, int NS, int D, bool grad) {
    LaneScratch s;
    float* f = reinterpret_cast<float*>(base);
    s.fr = f;
    f += kCostSlots * 12 * (NJ - 1);
    s.bc = f;
    f += kCostSlots * 3 * NJ;
    s.pos = f;
    f += kCostSlots * 3 * NS;
    s.dq = grad ? f : nullptr;
    if (grad) f += kCostSlots * NJ;
    s.q = f;
    f += kCostSlots * D;
    s.sc = f;
    f += kCostSlots * 2 * D;
    s.cand = reinterpret_cast<uint16_t*>(f);
    return s;
}

// Stages DoF d of the slot's waypoint, with its sine and cosine: the lanes of
// a group split the DoFs, so each angle's sincosf runs once per waypoint and
// the FK of every lane of the group reads it (a __syncwarp follows).
__device__ __forceinline__ void lane_put_q(const LaneScratch& ws, int slot, int d, float v) {
    float sn, cs;
    sincosf(v, &sn, &cs);
    ws.q[d * kCostSlots + slot] = v;
    ws.sc[(2 * d) * kCostSlots + slot] = sn;
    ws.sc[(2 * d + 1) * kCostSlots + slot] = cs;
}

// Bytes of a lane cost block: model core, staged scene, block tables, the
// warps' scratch.
inline size_t lane_block_bytes(const ps_model* m, const ps_scene_view* sv, int warps, bool grad) {
    return (size_t)m->dev.bytes_core + scene_smem_bytes(sv) + (((size_t)m->info.n_spheres + 15) & ~size_t(15)) + 64 +
           (size_t)16 * std::max(sv->n_obbs, 1) +
           (size_t)warps * lane_warp_bytes(m->info.n_joints, m->info.n_spheres, m->info.n_dof, sv->n_obbs, grad);
}

__device__ __forceinline__ void lane_frame(const float* fr, int p, int slot, Affine& T) {
    if (p == 0) {
        affine_identity(T);
        return;
    }
    const float* b = fr + (size_t)(p - 1) * 12 * kCostSlots + slot;
#pragma unroll
    for (int k = 0; k < 12; ++k) T.m[k] = b[k * kCostSlots];
}

// dC/dq_p of a summed force F and moment M (about the world origin) applied
// through joint j, added to every movable ancestor p of j (j included).
__device__ __forceinline__ void lane_fold(const ModelSmem& M, const LaneScratch& ws, int slot, int j, float Fx,
                                          float Fy, float Fz, float Mx, float My, float Mz) {
    for (int p = j; p >= 1; p = M.J[p].parent_pos) {
        const JointRec& jr = M.J[p];
        if (jr.dof < 0 || jr.type == PS_FIXED) continue;
        const float* b = ws.fr + (size_t)(p - 1) * 12 * kCostSlots + slot;
        const int ax = jr.type >= PS_X_ROT ? jr.type - PS_X_ROT : jr.type;
        const float axx = b[ax * kCostSlots], axy = b[(4 + ax) * kCostSlots], axz = b[(8 + ax) * kCostSlots];
        float v;
        if (jr.type >= PS_X_ROT) {
            const float ox = b[3 * kCostSlots], oy = b[7 * kCostSlots], oz = b[11 * kCostSlots];
            const float tx = Mx - (oy * Fz - oz * Fy);
            const float ty = My - (oz * Fx - ox * Fz);
            const float tz = Mz - (ox * Fy - oy * Fx);
            v = axx * tx + axy * ty + axz * tz;
        } else {
            v = axx * Fx + axy * Fy + axz * Fz;
        }
        ws.dq[p * kCostSlots + slot] += v;
    }
}

// Sum over the kCostSub lanes of a waypoint's group (fixed xor order).
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = 1; o < kCostSub; o <<= 1) v += __shfl_xor_sync(kCostFull, v, o);
    return v;
}

// Closest-box key of kG spheres over the candidate boxes: d^2 outside, the
// (non-positive) largest max(q) inside, i.e. d^2 + min(max(q), 0), exact in
// both cases. arg: the first candidate reaching the minimum (gradient only).
template <int kG, bool kGrad>
__device__ __forceinline__ void lane_keys(const SceneSmem& sc, const uint16_t* cand, int ncand, const float* px,
                                          const float* py, const float* pz, float* key, int* arg) {
#pragma unroll
    for (int i = 0; i < kG; ++i) {
        key[i] = 3.0e38f;
        arg[i] = -1;
    }
#pragma unroll 1
    for (int c = 0; c < ncand; ++c) {
        const int o = cand[c];
        const ObbPrep& b = sc.obbs[o];
        const float4 r0 = b.r0, r1 = b.r1, r2 = b.r2, h = b.h;
#pragma unroll
        for (int i = 0; i < kG; ++i) {
            const float lx = fmaf(r0.z, pz[i], fmaf(r0.y, py[i], fmaf(r0.x, px[i], r0.w)));
            const float ly = fmaf(r1.z, pz[i], fmaf(r1.y, py[i], fmaf(r1.x, px[i], r1.w)));
            const float lz = fmaf(r2.z, pz[i], fmaf(r2.y, py[i], fmaf(r2.x, px[i], r2.w)));
            const float qx = fabsf(lx) - h.x, qy = fabsf(ly) - h.y, qz = fabsf(lz) - h.z;
            const float cx = fmaxf(qx, 0.0f), cy = fmaxf(qy, 0.0f), cz = fmaxf(qz, 0.0f);
            const float k = fmaf(cz, cz, fmaf(cy, cy, cx * cx)) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
            if (kGrad) {
                if (k < key[i]) {
                    key[i] = k;
                    arg[i] = o;
                }
            } else {
                key[i] = fminf(key[i], k);
            }
        }
    }
}

// kN spheres of one lane: k0, k0 + kCostSub, ... (those at or past kend are
// marked invalid and replaced by k0), their world centres, radii and, over
// the candidate boxes, their closest-box keys. Slots kN..3 are invalid.
template <int kN, bool kGrad>
__device__ __forceinline__ void lane_group(const ModelSmem& M, const Affine& T, int k0, int kend,
                                           const SceneSmem& sc, const uint16_t* cand, int ncand, float* px, float* py,
                                           float* pz, float* rr, float* key, int* arg, int* kk, bool* val) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        key[i] = 3.0e38f;
        arg[i] = -1;
        val[i] = false;
        kk[i] = k0;
    }
#pragma unroll
    for (int i = 0; i < kN; ++i) {
        const int k = k0 + kCostSub * i;
        val[i] = k < kend;
        kk[i] = val[i] ? k : k0;
        const float4 sp = M.S[kk[i]];
        sphere_world(T, sp.x, sp.y, sp.z, px[i], py[i], pz[i]);
        rr[i] = sp.w;
    }
    if (ncand > 0) lane_keys<kN, kGrad>(sc, cand, ncand, px, py, pz, key, arg);
}

// Same for one sphere with its ACM row (global memory): masked boxes skipped.
__device__ __forceinline__ void lane_key_masked(const SceneSmem& sc, const uint16_t* cand, int ncand, float px,
                                                float py, float pz, const uint8_t* acm_row, float& key, int& arg) {
    key = 3.0e38f;
    arg = -1;
#pragma unroll 1
    for (int c = 0; c < ncand; ++c) {
        const int o = cand[c];
        if (acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        const float d2 = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        const float k = d2 + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
        if (k < key) {
            key = k;
            arg = o;
        }
    }
}

// Hinge terms of one sphere (box key already found): adds the OBB and ESDF
// hinges to the lane's partial sums and, with kGrad, returns the force on the
// sphere in (gx, gy, gz).
template <bool kGrad, bool kStats>
__device__ __forceinline__ void lane_sphere_terms(const ModelSmem& M, const SceneSmem& sc, const ps_scene_view& sv,
                                                  const ps_cost_params& P, int k, float px, float py, float pz,
                                                  float r, bool have_key, float key, int arg, float& obb_part,
                                                  float& esdf_part, float& gx, float& gy, float& gz, LaneStats& st) {
    const float w = P.collision_cost_weight, wm = P.world_margin;
    gx = gy = gz = 0.0f;
    if (have_key && key < 3.0e38f) {
        const float sdf = key > 0.0f ? sqrtf(key) : key;
        const float hinge = wm - (sdf - r);
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
    if (sc.n_layers) {
        const int so = M.SO[k];
        const uint8_t* eacm = sv.sphere_acm_mask ? sv.sphere_acm_mask + (size_t)so * sv.n_voxel_layers : nullptr;
        if (sv.esdf_mode == PS_ESDF_TRILINEAR) {
            // min over layers of -d - r; d(cost)/dp = w * grad d of the minimising layer
            float best = 1000.0f, bgx = 0.f, bgy = 0.f, bgz = 0.f;
            for (int l = 0; l < sc.n_layers; ++l) {
                if (eacm && eacm[l] == 0) continue;
                float d, dgx, dgy, dgz;
                if (kStats) st.v[ST_ESDF] += 1;
                if (!esdf_sample_trilinear_grad(sc.layers[l], sv.voxel_features + (size_t)l * sv.max_voxels_per_layer,
                                                sv.max_voxels_per_layer, px, py, pz, d, dgx, dgy, dgz))
                    continue;
                const float c = -d - r;
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
            LaneStats est;
            est.zero();
            const float clr = sphere_esdf_clearance(sc, sv, px, py, pz, r, eacm, est);
            if (kStats) st.v[ST_ESDF] += est.v[ST_ESDF];
            esdf_part += fmaxf(0.0f, wm - clr);
            // the nearest-voxel lookup is piecewise constant: zero gradient
        }
    }
}

// Cost of the lane group's waypoint (its configuration in ws.q) and, with
// kGrad, the per-joint gradient in ws.dq. Every lane of the warp calls it; the
// result is the same on the kCostSub lanes of a group.
template <bool kGrad, bool kStats>
__device__ float lane_cost(const ModelSmem& M, const ModelDev& md, const SceneSmem& sc, const ps_scene_view& sv,
                           const ps_cost_params& P, const CostBlock& cb, const LaneScratch& ws, LaneStats& st) {
    const float4* __restrict__ obs = cb.obs;
    const int lane = threadIdx.x & 31, slot = lane / kCostSub, u = lane % kCostSub;
    const int NJ = M.H->n_joints;
    const float w = P.collision_cost_weight, wmp = fmaxf(P.world_margin, 0.0f);
    float obb_part = 0.0f, esdf_part = 0.0f;
    if (kGrad && u == 0)
        for (int p = 0; p < NJ; ++p) ws.dq[p * kCostSlots + slot] = 0.0f;
    const bool masked = sv.sphere_obb_acm_mask != nullptr;
    Affine T;
    for (int p = 0; p < NJ; ++p) {
        const JointRec& jr = M.J[p];
        if (p == 0) {
            affine_identity(T);
        } else {
            const int dof = jr.dof;
            float qi = 0.0f, sn = 0.0f, cs = 1.0f;   // sincosf(0) for a joint without a DoF
            if (dof >= 0) {
                qi = ws.q[dof * kCostSlots + slot];
                sn = ws.sc[(2 * dof) * kCostSlots + slot];
                cs = ws.sc[(2 * dof + 1) * kCostSlots + slot];
            }
            if (jr.parent_pos == p - 1) {
                // the parent is the previous joint, whose frame is still in T (the
                // compose reads each parent row before writing it): no shared-memory
                // round trip on the chain's critical path
                joint_compose_sc(jr, qi, sn, cs, T, T);
            } else {
                Affine Pf;
                lane_frame(ws.fr, jr.parent_pos, slot, Pf);
                joint_compose_sc(jr, qi, sn, cs, Pf, T);
            }
            if (u == 0) {
                float* b = ws.fr + (size_t)(p - 1) * 12 * kCostSlots + slot;
#pragma unroll
                for (int k = 0; k < 12; ++k) b[k * kCostSlots] = T.m[k];
            }
            if (kStats && u == 0) st.v[ST_JOINTS] += 1;
        }
        __syncwarp();
        if (jr.bound.w < 0.0f) continue;   // no spheres on this joint (uniform)
        float cx, cy, cz;
        sphere_world(T, jr.bound.x, jr.bound.y, jr.bound.z, cx, cy, cz);
        if (u == 0) {
            ws.bc[(p * 3 + 0) * kCostSlots + slot] = cx;
            ws.bc[(p * 3 + 1) * kCostSlots + slot] = cy;
            ws.bc[(p * 3 + 2) * kCostSlots + slot] = cz;
        }
        const int n = jr.sph_end - jr.sph_beg;
        if (n == 0) continue;   // approximate spheres only: no cost term
        // ---- warp broad phase over boxes ----
        int ncand = 0;
        if (sc.n_obbs > 0) {
            const float mx = __shfl_sync(kCostFull, cx, 16), my = __shfl_sync(kCostFull, cy, 16),
                        mz = __shfl_sync(kCostFull, cz, 16);
            const float dx = cx - mx, dy = cy - my, dz = cz - mz;
            const float r2 =
                __uint_as_float(__reduce_max_sync(kCostFull, __float_as_uint(fmaf(dz, dz, fmaf(dy, dy, dx * dx)))));
            const float Sm = fmaxf(fabsf(mx), fmaxf(fabsf(my), fabsf(mz)));
            const float r2c = fmaxf(r2, 1.0e-30f);
            float Rc = r2c * rsqrtf(r2c) * (1.0f + 1.0e-6f) + jr.bound.w + wmp;
            Rc += 4.0f * (Sm + Rc + sc.Bmax + 1.0f) * PS_GUARD_K;
            const float Rcl = Rc * sc.Mscale;   // world radius -> box-frame radius (map stretch)
            const float Rc2 = Rcl * Rcl;
            const float Rj = (Rc * (1.0f + 4.0f * PS_GUARD_K) + 4.0f * PS_GUARD_K * (Sm + 1.0f)) * (1.0f + 1.0e-6f);
            __syncwarp();   // the previous joint's readers of ws.cand are done
#pragma unroll 1
            for (int base = 0; base < sc.n_obbs; base += 32) {
                const int o = base + lane;
                bool keep = false;
                if (o < sc.n_obbs) {
                    const float4 ob = obs[o];
                    const float ex = ob.x - mx, ey = ob.y - my, ez = ob.z - mz;
                    const float lim = Rj + ob.w;   // split guarded limit (box_limits)
                    if (fmaf(ez, ez, fmaf(ey, ey, ex * ex)) < lim * lim) {
                        float qx, qy, qz;
                        keep = fast_box_dsq(sc.obbs[o], mx, my, mz, qx, qy, qz) < Rc2;
                    }
                    if (kStats) st.v[ST_CULL] += 1;
                }
                const unsigned bal = __ballot_sync(kCostFull, keep);
                if (keep) ws.cand[ncand + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)o;
                ncand += __popc(bal);
            }
            __syncwarp();
        }
        // ---- the joint's spheres: lane u of the group takes spheres
        //      sph_beg + u, + kCostSub, ... (up to 4 per box load) ----
        float Fx = 0.f, Fy = 0.f, Fz = 0.f, Mx = 0.f, My = 0.f, Mz = 0.f;
        const int nm = (n + kCostSub - 1) / kCostSub;   // spheres per lane, uniform
        for (int m0 = 0; m0 < nm;) {
            const int ng = masked ? 1 : min(4, nm - m0);   // uniform
            float px[4], py[4], pz[4], rr[4], key[4];
            int arg[4], kk[4];
            bool val[4];
            const int k0 = jr.sph_beg + u + kCostSub * m0;
            if (ng == 4)
                lane_group<4, kGrad>(M, T, k0, jr.sph_end, sc, ws.cand, ncand, px, py, pz, rr, key, arg, kk, val);
            else if (ng == 3)
                lane_group<3, kGrad>(M, T, k0, jr.sph_end, sc, ws.cand, ncand, px, py, pz, rr, key, arg, kk, val);
            else if (ng == 2)
                lane_group<2, kGrad>(M, T, k0, jr.sph_end, sc, ws.cand, ncand, px, py, pz, rr, key, arg, kk, val);
            else if (!masked)
                lane_group<1, kGrad>(M, T, k0, jr.sph_end, sc, ws.cand, ncand, px, py, pz, rr, key, arg, kk, val);
            else {
                lane_group<1, kGrad>(M, T, k0, jr.sph_end, sc, ws.cand, 0, px, py, pz, rr, key, arg, kk, val);
                if (ncand > 0)
                    lane_key_masked(sc, ws.cand, ncand, px[0], py[0], pz[0],
                                    sv.sphere_obb_acm_mask + (size_t)M.SO[kk[0]] * sv.n_obbs, key[0], arg[0]);
            }
            if (kStats)
                for (int i = 0; i < 4; ++i)
                    if (val[i]) {
                        st.v[ST_SPHERES] += 1;
                        st.v[ST_PAIRS] += ncand;
                    }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (!val[i]) continue;
                ws.pos[(kk[i] * 3 + 0) * kCostSlots + slot] = px[i];
                ws.pos[(kk[i] * 3 + 1) * kCostSlots + slot] = py[i];
                ws.pos[(kk[i] * 3 + 2) * kCostSlots + slot] = pz[i];
                float gx, gy, gz;
                lane_sphere_terms<kGrad, kStats>(M, sc, sv, P, kk[i], px[i], py[i], pz[i], rr[i], ncand > 0, key[i],
                                                 arg[i], obb_part, esdf_part, gx, gy, gz, st);
                if (kGrad) {
                    Fx += gx;
                    Fy += gy;
                    Fz += gz;
                    Mx += py[i] * gz - pz[i] * gy;
                    My += pz[i] * gx - px[i] * gz;
                    Mz += px[i] * gy - py[i] * gx;
                }
            }
            m0 += ng;
        }
        if (kGrad) {
            Fx = group_sum(Fx);
            Fy = group_sum(Fy);
            Fz = group_sum(Fz);
            Mx = group_sum(Mx);
            My = group_sum(My);
            Mz = group_sum(Mz);
            const bool any = Fx != 0.f || Fy != 0.f || Fz != 0.f || Mx != 0.f || My != 0.f || Mz != 0.f;
            if (__any_sync(kCostFull, any) && u == 0) lane_fold(M, ws, slot, p, Fx, Fy, Fz, Mx, My, Mz);
        }
    }
    __syncwarp();   // frames and bound centres of every joint are written

    // ---- self hinge ----
    float self_h = 0.0f;
    if (P.include_self && md.n_sjp > 0) {
        const float smg = P.self_margin, smp = fmaxf(smg, 0.0f);
        float bv = smg;   // pairs at or above the margin cannot set the hinge
        int bk = INT_MAX, bi = -1, bj = -1;
        // cull level: the smallest clearance the group has found (at most bv).
        // A pair or run that cannot come below it cannot set the group's
        // minimum; the joint pairs come nearest first, so it drops early.
        float cl = smg;
        auto at = [&](const float* a, int k, int c) { return a[(k * 3 + c) * kCostSlots + slot]; };
        for (int jp0 = 0; jp0 < md.n_sjp; jp0 += kCostSub) {
            cl = fminf(cl, __shfl_xor_sync(kCostFull, cl, 1));
            cl = fminf(cl, __shfl_xor_sync(kCostFull, cl, 2));
            // lane u tests joint pair jp0 + u on its own waypoint; one ballot
            // gives each pair's OR over the warp's waypoints
            bool pass = false;
            if (jp0 + u < md.n_sjp) {
                const uint4 e = __ldg(md.sjp + jp0 + u);
                const int a = (int)(e.x & 0xffffu), qj = (int)(e.x >> 16);
                const float ax = at(ws.bc, a, 0), ay = at(ws.bc, a, 1), az = at(ws.bc, a, 2);
                const float qx0 = at(ws.bc, qj, 0), qy0 = at(ws.bc, qj, 1), qz0 = at(ws.bc, qj, 2);
                const float dx = ax - qx0, dy = ay - qy0, dz = az - qz0;
                const float S = fmaxf(fmaxf(fabsf(ax), fmaxf(fabsf(ay), fabsf(az))),
                                      fmaxf(fabsf(qx0), fmaxf(fabsf(qy0), fabsf(qz0))));
                const float rr = M.J[a].bound.w + M.J[qj].bound.w;
                // clearance of any pair >= |c_a - c_q| - R_a - R_q, plus a guard for the FP32 centres
                const float thr = rr + cl + 4.0f * (S + rr + smp + 1.0f) * PS_GUARD_K;
                pass = thr > 0.0f && fmaf(dz, dz, fmaf(dy, dy, dx * dx)) < thr * thr;
                if (kStats) st.v[ST_SELF] += 1;
            }
            const unsigned bal = __ballot_sync(kCostFull, pass);
            for (int v = 0; v < kCostSub && jp0 + v < md.n_sjp; ++v) {
                if (!(bal & (0x11111111u << v))) continue;   // uniform
                const uint4 e = __ldg(md.sjp + jp0 + v);
                const int a = (int)(e.x & 0xffffu), qj = (int)(e.x >> 16);
                const float Ra = M.J[a].bound.w, Rq = M.J[qj].bound.w;
                const float cqx = at(ws.bc, qj, 0), cqy = at(ws.bc, qj, 1), cqz = at(ws.bc, qj, 2);
                // run reach: clearance of sphere i against any sphere of q >= |p_i - c_q| - R_q - r_i;
                // the guard covers the FP32 centres, from bounds that hold for every sphere i of joint a
                const float Sjp = fmaxf(fmaxf(fabsf(at(ws.bc, a, 0)), fmaxf(fabsf(at(ws.bc, a, 1)),
                                                                            fabsf(at(ws.bc, a, 2)))) + Ra,
                                        fmaxf(fabsf(cqx), fmaxf(fabsf(cqy), fabsf(cqz))));
                const float reach = Rq + 4.0f * (Sjp + Ra + Rq + smp + 1.0f) * PS_GUARD_K;
                // the group's lanes split the runs; a lane tests its run on its own waypoint
                for (int r0 = (int)e.y; r0 < (int)e.z; r0 += kCostSub) {
                    const int r = r0 + u;
                    if (r >= (int)e.z) continue;
                    const uint2 run = __ldg(md.sruns + r);
                    const int i = run.x & 0x1ffu, len = (run.x >> 14) & 0x1ffu, j0 = (int)run.y;
                    const float ri = M.S[i].w;
                    const float pxi = at(ws.pos, i, 0), pyi = at(ws.pos, i, 1), pzi = at(ws.pos, i, 2);
                    const float ex = pxi - cqx, ey = pyi - cqy, ez = pzi - cqz;
                    const float rt = ri + reach + cl;
                    if (kStats) st.v[ST_SELF] += 1;
                    if (rt <= 0.0f || fmaf(ez, ez, fmaf(ey, ey, ex * ex)) >= rt * rt) continue;   // none gets below cl
                    // sqrt(d2) - (ri + rj) <= cl needs sqrt(d2) <= cl + ri + rj; the bound t
                    // adds 2e-6 (|cl| + ri + rj), some 16 ulps of every term that rounds in
                    // either expression, so a pair at the cull level itself (a tie with a
                    // pair another lane found) is never rejected here, however close its
                    // centres. When t <= 0 no pair gets below cl and the test passes at most
                    // pairs that the exact test then keeps out of the group minimum.
                    float tb = cl + ri + 2.0e-6f * (fabsf(cl) + ri);
#pragma unroll 4
                    for (int m = 0; m < len; ++m) {
                        const int j = j0 + m;
                        const float vx = pxi - at(ws.pos, j, 0), vy = pyi - at(ws.pos, j, 1),
                                    vz = pzi - at(ws.pos, j, 2);
                        const float d2 = fmaf(vz, vz, fmaf(vy, vy, vx * vx));
                        const float rj = M.S[j].w;
                        const float t = fmaf(rj, 1.000002f, tb);
                        if (d2 * (1.0f - 4.0e-6f) < t * t) {   // can get below cl: take the root
                            const float c = sqrtf(d2) - (ri + rj);
                            const int key = (r << 9) | m;
                            if (c < bv || (c == bv && key < bk)) {
                                bv = c;
                                bk = key;
                                bi = i;
                                bj = j;
                                cl = fminf(cl, c);
                                tb = cl + ri + 2.0e-6f * (fabsf(cl) + ri);
                            }
                        }
                    }
                    if (kStats) st.v[ST_SELF] += len;
                }
            }
        }
        // minimum over the group by (value, pair order)
#pragma unroll
        for (int o = 1; o < kCostSub; o <<= 1) {
            const float ov = __shfl_xor_sync(kCostFull, bv, o);
            const int ok = __shfl_xor_sync(kCostFull, bk, o);
            const int oi = __shfl_xor_sync(kCostFull, bi, o);
            const int oj = __shfl_xor_sync(kCostFull, bj, o);
            if (ov < bv || (ov == bv && ok < bk)) {
                bv = ov;
                bk = ok;
                bi = oi;
                bj = oj;
            }
        }
        self_h = fmaxf(0.0f, smg - bv);
        if (kGrad && u == 0 && bi >= 0 && self_h > 0.0f) {
            // world positions of the pair: d self_h / d p_i = -(p_i - p_j) / |p_i - p_j|
            const int pi = cb.sph_joint[bi], pj = cb.sph_joint[bj];
            const float xi = at(ws.pos, bi, 0), yi = at(ws.pos, bi, 1), zi = at(ws.pos, bi, 2);
            const float xj = at(ws.pos, bj, 0), yj = at(ws.pos, bj, 1), zj = at(ws.pos, bj, 2);
            const float dx = xi - xj, dy = yi - yj, dz = zi - zj;
            const float dd = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
            if (dd > 0.0f) {
                const float s = w / dd;
                const float gx = -s * dx, gy = -s * dy, gz = -s * dz;   // on p_i; -g on p_j
                lane_fold(M, ws, slot, pi, gx, gy, gz, yi * gz - zi * gy, zi * gx - xi * gz, xi * gy - yi * gx);
                lane_fold(M, ws, slot, pj, -gx, -gy, -gz, -(yj * gz - zj * gy), -(zj * gx - xj * gz),
                          -(xj * gy - yj * gx));
            }
        }
    }
    if (kGrad) __syncwarp();   // the group leaders' folds are visible to lane_write_grad
    return w * (group_sum(esdf_part) + group_sum(obb_part) + self_h);
}

// d cost / d q per DoF from the per-joint gradient: a DoF's one joint, or the
// sum over the joints that share it (DFS order). The group's lanes write
// DoFs u, u + kCostSub, ... to row[d * stride].
__device__ __forceinline__ void lane_write_grad(const ModelSmem& M, const CostBlock& cb, const LaneScratch& ws,
                                                float* row, int stride) {
    const int lane = threadIdx.x & 31, slot = lane / kCostSub, u = lane % kCostSub;
    const int D = M.H->n_dof, NJ = M.H->n_joints;
    for (int d = u; d < D; d += kCostSub) {
        const int who = cb.dof_joint[d];
        float acc = 0.0f;
        if (who >= 0) {
            acc = ws.dq[who * kCostSlots + slot];
        } else if (who == -2) {
            for (int p = 1; p < NJ; ++p)
                if (M.J[p].dof == d && M.J[p].type != PS_FIXED) acc += ws.dq[p * kCostSlots + slot];
        }
        row[(size_t)d * stride] = acc;
    }
}

}  // namespace
}  // namespace ps
