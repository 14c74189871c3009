// ps_costwarp.cuh -- per-waypoint summed-hinge cost and its adjoint, one
// warp per waypoint. Shared by the trajectory kernels (ps_cost.cu) and the
// mixed-request batch (ps_batch.cu).
//
// Cost of one configuration (chomp.cu:151-188 / stomp.cu:206-245 over
// scene_collision.cuh:394-495 and runtime_kinematics.cuh:295-330):
//   w * ( sum_s relu(m - esdf_clr_s) + sum_s relu(m - min_o obb_clr_s,o)
//         + relu(m_self - min_(i,j) (|p_i - p_j| - r_i - r_j)) ).
// The reference evaluates every sphere against every box and every self pair
// in one thread. Here a warp takes a tile of kCostTile consecutive waypoints;
// steps 1 and 3-5 run per waypoint with the 32 lanes sharing it, step 2 once
// per tile:
//   1. FK: lane p evaluates joint p's sine/cosine, every lane walks the chain
//      with them, lane p keeps frame p in shared memory;
//   2. per joint, the boxes that can reach any of its spheres within the
//      hinge band are found from the union of the joint's bound spheres over
//      the tile's waypoints (lanes over boxes,
//      one ballot word per 32 boxes): a box farther than R_p + max(m, 0)
//      from the bound centre has sdf > m + r for every sphere of the joint
//      and contributes nothing. A circumscribed-sphere test of the box comes
//      first, the box distance only for the boxes it keeps;
//   3. lanes over spheres: closest candidate box, ESDF, hinge and d/dp;
//   4. self hinge: joint pairs whose bound spheres are within m_self of each
//      other expand their sphere pairs across the lanes; a pair whose squared
//      distance is outside (r_i + r_j + m_self)^2 cannot set the hinge and
//      skips the square root; warp argmin;
//   5. adjoint: per joint F = sum g, M = sum p x g (lane per joint), subtree
//      accumulation from the leaves, dC/dq = a . (M - o x F) (revolute) or
//      a . F (prismatic), a/o the joint axis/origin in the world.
// Sums run in a fixed order (lane-strided partials, xor-tree reduction), so a
// waypoint gives the same bits wherever it is evaluated.
#pragma once

#include <algorithm>
#include <cstdint>

#include "ps_internal.h"
#include "ps_verdict.cuh"

namespace ps {
namespace {

constexpr unsigned kCostFull = 0xffffffffu;

// Most waypoints per warp tile: the box cull of a joint is done once per
// tile, against the union of the joint's bound spheres over the tile's
// waypoints. Kernels run tiles of 1 or kCostTile waypoints.
constexpr int kCostTile = 4;

// Per-warp scratch in shared memory (floats unless noted; 16-byte aligned).
struct CostWarpScratch {
    float* q;        // [kCostTile][16]
    float* frame;    // [kCostTile][NJ][12]
    float4* bnd;     // [kCostTile][NJ]: bound centre (world), radius
    float4* ubnd;    // [NJ][2]: (union centre, -), (box cull threshold, its square, |centre|inf, -)
    float4* pos;     // [NS]: centre (world), radius
    float* g;        // [NS][3]   (gradient only)
    float* jfm;      // [NJ][8]: F, M, dC/dq   (gradient only)
    unsigned* mask;  // [NJ][nw]  candidate boxes per joint
    uint16_t* alist; // [n_sruns] active self-pair runs
};

__host__ __device__ inline int cost_mask_words(int n_obbs) { return (n_obbs + 31) / 32; }

__host__ __device__ inline size_t cost_warp_floats(int NJ, int NS, int n_obbs, int n_sruns, bool grad) {
    size_t f = (size_t)kCostTile * (16 + (size_t)NJ * 12 + (size_t)NJ * 4) + (size_t)NJ * 8 + (size_t)NS * 4;
    if (grad) f += (size_t)NS * 3 + (size_t)NJ * 8;
    f = (f + 3) & ~size_t(3);
    f += (size_t)NJ * cost_mask_words(n_obbs) + ((size_t)n_sruns + 1) / 2;
    return (f + 3) & ~size_t(3);   // keep every warp's slice 16-byte aligned
}

__device__ __forceinline__ CostWarpScratch cost_carve(float* base, int NJ, int NS, int n_obbs, bool grad) {
    CostWarpScratch w;
    w.q = base;
    w.frame = w.q + kCostTile * 16;
    w.bnd = reinterpret_cast<float4*>(w.frame + kCostTile * NJ * 12);
    w.ubnd = w.bnd + kCostTile * NJ;
    w.pos = w.ubnd + NJ * 2;
    float* p = reinterpret_cast<float*>(w.pos + NS);
    if (grad) {
        w.g = p;
        w.jfm = w.g + NS * 3;
        p = w.jfm + NJ * 8;
    } else {
        w.g = nullptr;
        w.jfm = nullptr;
    }
    p = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
    w.mask = reinterpret_cast<unsigned*>(p);
    w.alist = reinterpret_cast<uint16_t*>(w.mask + NJ * cost_mask_words(n_obbs));
    return w;
}

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

inline size_t cost_block_bytes(const ps_model* m, const ps_scene_view* sv, int warps, bool grad) {
    return (size_t)m->dev.bytes_core + scene_smem_bytes(sv) + (((size_t)m->info.n_spheres + 15) & ~size_t(15)) + 64 +
           (size_t)16 * std::max(sv->n_obbs, 1) +
           (size_t)warps * cost_warp_floats(m->info.n_joints, m->info.n_spheres, sv->n_obbs, m->dev.n_sruns, grad) * 4;
}

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

// FK of the nt waypoints of a tile: frames and world bound spheres of every
// joint. The warp splits into groups of n_joints lanes, one group per
// waypoint (32 / n_joints waypoints per pass). In a group, lane p forms joint
// p's local step S_p = FT_p * motion(q) with accurate sincosf and holds A_p,
// the transform from its current ancestor anc_p to p; each round composes
// A_anc * A_p and jumps anc_p to anc_anc, so depth d takes ceil(log2 d)
// rounds. A frame's factors and their order depend only on the tree, so a
// waypoint gets the same bits in any group and tile.
template <bool kStats>
__device__ __forceinline__ void cost_fk_tile(const ModelSmem& M, const float* q, int nt, float* frame, float4* bnd,
                                             LaneStats& st) {
    const int lane = threadIdx.x & 31;
    const int NJ = M.H->n_joints;
    const int per = max(1, 32 / NJ);
    const int grp = lane / NJ, p = lane - grp * NJ, base = grp * NJ;
    for (int t0 = 0; t0 < nt; t0 += per) {
        const int t = t0 + grp;
        const bool act = grp < per && t < nt;
        Affine A;
        affine_identity(A);
        int anc = -1;
        if (act && p > 0) {
            const JointRec& jr = M.J[p];
            const float qi = jr.dof >= 0 ? q[t * 16 + jr.dof] : 0.0f;
            float sn = 0.0f, cs = 1.0f;
            if (jr.type >= PS_X_ROT) sincosf(qi, &sn, &cs);
            Affine I;
            affine_identity(I);
            joint_compose_sc(jr, qi, sn, cs, I, A);
            anc = jr.parent_pos;
        }
        while (__ballot_sync(kCostFull, anc >= 0)) {
            const int src = anc >= 0 ? base + anc : lane;
            Affine B;
#pragma unroll
            for (int i = 0; i < 12; ++i) B.m[i] = __shfl_sync(kCostFull, A.m[i], src);
            const int anc2 = __shfl_sync(kCostFull, anc, src);
            if (anc >= 0) {
                Affine C;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        float v = fmaf(B.m[r * 4 + 2], A.m[8 + c], fmaf(B.m[r * 4 + 1], A.m[4 + c], B.m[r * 4] * A.m[c]));
                        C.m[r * 4 + c] = c == 3 ? v + B.m[r * 4 + 3] : v;
                    }
                }
                A = C;
                anc = anc2;
            }
        }
        if (act) {
            store_frame(frame + ((size_t)t * NJ + p) * 12, A);
            const float4 b = M.J[p].bound;
            float cx = 0.f, cy = 0.f, cz = 0.f;
            if (b.w >= 0.0f) sphere_world(A, b.x, b.y, b.z, cx, cy, cz);
            bnd[t * NJ + p] = make_float4(cx, cy, cz, b.w);
        }
    }
    if (kStats && lane == 0) st.v[ST_JOINTS] += NJ * nt;
    __syncwarp();
}

// Candidate boxes per joint for a tile of nt waypoints, from the union of
// the joint's bound spheres over the tile: a box farther than that union's
// radius + max(m, 0) reaches no sphere of the joint inside the hinge band.
template <bool kStats>
__device__ __forceinline__ void cost_cull(const ModelSmem& M, const SceneSmem& sc, const CostBlock& cb,
                                          const CostWarpScratch& ws, int nt, float wm, LaneStats& st) {
    const int lane = threadIdx.x & 31;
    const int NJ = M.H->n_joints;
    const int nob = sc.n_obbs, nw = cost_mask_words(nob);
    for (int p = lane; p < NJ; p += 32) {
        const float4 c0 = ws.bnd[p];
        float thr = -1.0f, S = 0.0f;
        if (c0.w >= 0.0f) {
            float r2 = 0.0f;
            for (int t = 1; t < nt; ++t) {
                const float4 c = ws.bnd[t * NJ + p];
                const float dx = c.x - c0.x, dy = c.y - c0.y, dz = c.z - c0.z;
                r2 = fmaxf(r2, fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
            }
            // slack for the FP32 rounding of the transforms and the tests
            S = fmaxf(fabsf(c0.x), fmaxf(fabsf(c0.y), fabsf(c0.z)));
            thr = sqrtf(r2) + c0.w + fmaxf(wm, 0.0f);
            thr += 4.0f * (S + thr + sc.Bmax + 1.0f) * PS_GUARD_K;
        }
        ws.ubnd[p * 2] = make_float4(c0.x, c0.y, c0.z, c0.w);
        ws.ubnd[p * 2 + 1] = make_float4(thr, thr * thr, S, 0.0f);
    }
    __syncwarp();
    // ---- 2. candidate boxes per joint (lanes over boxes): circumscribed-
    //      sphere prefilter, then the box distance of the bound centre ----
    if (nob > 0) {
        for (int base = 0; base < nob; base += 32) {
            const int o = base + lane;
            const bool ok = o < nob;
            float4 ob = make_float4(0.f, 0.f, 0.f, -1.0f);
            if (ok) ob = cb.obs[o];
            const float So = fmaxf(fabsf(ob.x), fmaxf(fabsf(ob.y), fabsf(ob.z))) + ob.w;
            const int njs = *cb.njs;
            for (int pi = 0; pi < njs; ++pi) {
                const int p = cb.jlist[pi];
                const float4 bc = ws.ubnd[p * 2];
                const float4 th = ws.ubnd[p * 2 + 1];
                bool keep = false;
                if (ok && bc.w >= 0.0f) {
                    const float dx = bc.x - ob.x, dy = bc.y - ob.y, dz = bc.z - ob.z;
                    float lim = th.x + ob.w;
                    lim += 4.0f * (So + th.z + lim + 1.0f) * PS_GUARD_K;
                    if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) < lim * lim) {
                        float qx, qy, qz;
                        keep = fast_box_dsq(sc.obbs[o], bc.x, bc.y, bc.z, qx, qy, qz) < th.y;
                    }
                    if (kStats) st.v[ST_CULL] += 1;
                }
                const unsigned bal = __ballot_sync(kCostFull, keep);
                if (lane == 0) ws.mask[p * nw + (base >> 5)] = bal;
            }
        }
        __syncwarp();
    }
}

// Cost (returned on every lane) of waypoint t of the tile and, with kGrad,
// d cost / d q written by lanes d < n_dof to grad_row[d * gstride]. The whole
// warp calls it after cost_fk_tile and cost_cull. kStats: count executed work.
template <bool kGrad, bool kStats>
__device__ __forceinline__ float cost_eval(const ModelSmem& M, const ModelDev& md, const SceneSmem& sc,
                                           const ps_scene_view& sv, const ps_cost_params& P, const CostBlock& cb,
                                           const CostWarpScratch& ws, int t, float* grad_row, int gstride,
                                           LaneStats& st) {
    const int lane = threadIdx.x & 31;
    const int D = M.H->n_dof, NJ = M.H->n_joints, NS = M.H->n_spheres;
    const float w = P.collision_cost_weight, wm = P.world_margin, smg = P.self_margin;
    const int nob = sc.n_obbs, nw = cost_mask_words(nob);
    const float* fr = ws.frame + t * NJ * 12;
    const float4* bw = ws.bnd + t * NJ;
    // ---- 3. spheres (lanes over spheres) ----
    float obb_part = 0.0f, esdf_part = 0.0f;
    for (int k = lane; k < NS; k += 32) {
        const int p = cb.sph_joint[k];
        const float4 sp = M.S[k];
        Affine T;
        load_frame(fr + p * 12, T);
        float px, py, pz;
        sphere_world(T, sp.x, sp.y, sp.z, px, py, pz);
        ws.pos[k] = make_float4(px, py, pz, sp.w);
        if (kStats) st.v[ST_SPHERES] += 1;
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
            if (kStats) st.v[ST_PAIRS] += tests;
        }
        if (sc.n_layers) {
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
                LaneStats est;
                est.zero();
                const float clr = sphere_esdf_clearance(sc, sv, px, py, pz, sp.w, eacm, est);
                if (kStats) st.v[ST_ESDF] += est.v[ST_ESDF];
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

    // ---- 4. self hinge. A run (sphere i against the spheres of joint q) can
    //      hold a pair with |p_i - p_j| - r_i - r_j < m_self only if
    //      |p_i - c_q| < r_i + R_q + m_self: lanes test the runs, ballot-
    //      compact the active ones, then each lane walks whole active runs. ----
    float self_h = 0.0f;
    int self_i = -1, self_j = -1;
    if (P.include_self && md.n_sruns > 0) {
        const float smp = fmaxf(smg, 0.0f);
        int n_act = 0;
        for (int base = 0; base < md.n_sruns; base += 32) {
            const int r = base + lane;
            bool act = false;
            if (r < md.n_sruns) {
                const uint2 run = __ldg(md.sruns + r);
                const float4 a = ws.pos[run.x & 0x1ffu];
                const float4 c = bw[(run.x >> 9) & 31u];
                const float dx = a.x - c.x, dy = a.y - c.y, dz = a.z - c.z;
                const float S = fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fmaxf(fabsf(c.x),
                                fmaxf(fabsf(c.y), fabsf(c.z)))));
                float thr = a.w + c.w + smp;
                thr += 4.0f * (S + thr + 1.0f) * PS_GUARD_K;
                act = fmaf(dz, dz, fmaf(dy, dy, dx * dx)) < thr * thr;
                if (kStats) st.v[ST_SELF] += 1;
            }
            const unsigned bal = __ballot_sync(kCostFull, act);
            if (act) ws.alist[n_act + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)r;
            n_act += __popc(bal);
        }
        __syncwarp();
        float bv = 3.0e38f;
        int bk = 0x7fffffff, bi = -1, bj = -1;
        for (int t = lane; t < n_act; t += 32) {
            const uint2 run = __ldg(md.sruns + ws.alist[t]);
            const int i = run.x & 0x1ffu, len = (run.x >> 14) & 0x1ffu;
            const float4 a = ws.pos[i];
            for (int u = 0; u < len; ++u) {
                const int k = (int)run.y + u;
                const int j = __ldg(md.spairs + k);
                const float4 b = ws.pos[j];
                const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
                const float d2 = fmaxf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)), 1.0e-30f);
                const float c = d2 * rsqrtf(d2) - (a.w + b.w);
                if (kStats) st.v[ST_SELF] += 1;
                if (c < bv) {   // k increases along a lane: the first minimum wins ties
                    bv = c;
                    bk = k;
                    bi = i;
                    bj = j;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
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
        if (self_h > 0.0f) {
            self_i = bi;
            self_j = bj;
        }
    }
    const float cost = w * (warp_sum(esdf_part) + warp_sum(obb_part) + self_h);
    if (!kGrad) return cost;

    // ---- 5. adjoint ----
    if (self_i >= 0 && lane == 0) {
        const int i = self_i, j = self_j;
        const float4 a = ws.pos[i], b = ws.pos[j];
        const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
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
            const float4 pk = ws.pos[k];
            Fx += gx; Fy += gy; Fz += gz;
            Mx += pk.y * gz - pk.z * gy;
            My += pk.z * gx - pk.x * gz;
            Mz += pk.x * gy - pk.y * gx;
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
            const float* T = fr + p * 12;
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
    // lane d writes DoF d: its joint's term, or, for a DoF that drives several
    // joints, their sum in DFS order
    for (int d = lane; d < D; d += 32) {
        const int who = cb.dof_joint[d];
        float acc = 0.0f;
        if (who >= 0) {
            acc = ws.jfm[who * 8 + 6];
        } else if (who == -2) {
            for (int p = 1; p < NJ; ++p)
                if (M.J[p].dof == d && M.J[p].type != PS_FIXED) acc += ws.jfm[p * 8 + 6];
        }
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
