// ps_verdict.cuh -- per-lane collision verdicts (one configuration per lane).
//
// Semantics are two_phase_cc's (code/gpu_planning/cpp/src/collision/
// two_phase_cc.cuh:57-138) for one configuration: the approximate spheres of
// joint j are tested against the scene (OBBs + ESDF, radius + margin,
// scene_collision.cuh:584-631); if any hits, joint j is flagged and its exact
// spheres are tested (scene_collision.cuh:519-567). The configuration
// collides iff some exact sphere of a flagged joint hits. The order of the
// tests does not change that OR, so the kernels test joint by joint during the
// FK walk and stop at the first confirmed hit.
#pragma once

#include "ps_common.cuh"
#include "ps_stage.cuh"

namespace ps {

// Diagnostic counters (device, optional): executed work for the roofline.
enum StatSlot {
    ST_PAIRS = 0,        // sphere-vs-box pair tests (fast path)
    ST_EXACT = 1,        // pairs re-decided with the exact reference sequence
    ST_SAMPLES = 2,      // configurations / samples evaluated
    ST_JOINTS = 3,       // FK joint steps
    ST_SPHERES = 4,      // sphere transforms
    ST_SELF = 5,         // self pair tests
    ST_ESDF = 6,         // ESDF lookups
    ST_CULL = 7,         // broad-phase box tests
    ST_COUNT = 8
};

struct LaneStats {
    unsigned int v[ST_COUNT];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int k = 0; k < ST_COUNT; ++k) v[k] = 0;
    }
};

// Block-reduce the lane counters and add them with one atomic per slot.
__device__ __forceinline__ void flush_stats(unsigned long long* stats, LaneStats& ls) {
    if (!stats) return;
#pragma unroll
    for (int k = 0; k < ST_COUNT; ++k) {
        unsigned int x = ls.v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(stats + k, (unsigned long long)x);
    }
}

// Whether a sphere (centre c, radius R) can reach the voxel box of any
// enabled ESDF layer: its centre, mapped into the layer frame, within R (plus
// slack for the FP32 map) of the grid extent on every axis. A lookup outside
// the extent never reports a distance, so a sphere set inside that bound sees
// no layer.
__device__ __forceinline__ bool esdf_reachable(const SceneSmem& sc, float cx, float cy, float cz, float R) {
    for (int l = 0; l < sc.n_layers; ++l) {
        const LayerPrep& L = sc.layers[l];
        if (!L.enabled) continue;
        float lx, ly, lz;
        ref_to_local(L.q.x, L.q.y, L.q.z, L.q.w, L.t.x, L.t.y, L.t.z, cx, cy, cz, lx, ly, lz);
        const float S = fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz))) + fmaxf(fabsf(L.t.x), fmaxf(fabsf(L.t.y), fabsf(L.t.z)));
        const float Rl = R * sc.Mscale;   // a world distance R is at most R * Mscale in the layer frame
        const float slack = 1.0e-4f * (S + Rl + 1.0f);
        if (fabsf(lx) <= 0.5f * L.params.x + Rl + slack && fabsf(ly) <= 0.5f * L.params.y + Rl + slack &&
            fabsf(lz) <= 0.5f * L.params.z + Rl + slack)
            return true;
    }
    return false;
}

// World centre and circumscribed radius of each staged box: local = M p + t,
// so the centre is -M^-1 t (M^-1 from its adjugate) and the box's world points
// lie within |h| |M^-1| of it (quat_norm_err / map_stretch bound |M^-1|; a
// box outside that bound gets an unbounded radius). Every thread of the block
// calls it.
__device__ __forceinline__ void box_spheres(const SceneSmem& sc, float4* obs) {
    for (int o = threadIdx.x; o < sc.n_obbs; o += blockDim.x) {
        const ObbPrep& b = sc.obbs[o];
        const float e = quat_norm_err(b.q.x, b.q.y, b.q.z, b.q.w);
        const float lo = 1.0f - 4.0f * e * (1.0f + e);
        // adjugate columns: M^-1 = [r1 x r2, r2 x r0, r0 x r1] / det
        const float ax = b.r1.y * b.r2.z - b.r1.z * b.r2.y, ay = b.r1.z * b.r2.x - b.r1.x * b.r2.z,
                    az = b.r1.x * b.r2.y - b.r1.y * b.r2.x;
        const float bx = b.r2.y * b.r0.z - b.r2.z * b.r0.y, by = b.r2.z * b.r0.x - b.r2.x * b.r0.z,
                    bz = b.r2.x * b.r0.y - b.r2.y * b.r0.x;
        const float cx2 = b.r0.y * b.r1.z - b.r0.z * b.r1.y, cy2 = b.r0.z * b.r1.x - b.r0.x * b.r1.z,
                    cz2 = b.r0.x * b.r1.y - b.r0.y * b.r1.x;
        const float det = b.r0.x * ax + b.r0.y * ay + b.r0.z * az;
        float4 out;
        if (lo >= 0.25f && fabsf(det) > 0.25f) {
            const float inv = 1.0f / det;
            out.x = -(b.r0.w * ax + b.r1.w * bx + b.r2.w * cx2) * inv;
            out.y = -(b.r0.w * ay + b.r1.w * by + b.r2.w * cy2) * inv;
            out.z = -(b.r0.w * az + b.r1.w * bz + b.r2.w * cz2) * inv;
            out.w = sqrtf(b.h.x * b.h.x + b.h.y * b.h.y + b.h.z * b.h.z) * rsqrtf(lo) * (1.0f + 1.0e-5f);
        } else {
            out = make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);   // never culled by the prefilter
        }
        obs[o] = out;
    }
}

// Circumscribed-sphere prefilter of the fast path's broad phase. With
// Rc the joint's cull radius around the chunk centre m (Sm = |m|inf), box o's
// centre c_o (M_o = |c_o|inf) and circumscribed radius w_o, the guarded limit
//   Rc + w_o + 4K (Sm + M_o + Rc + w_o + 1)
// splits into a joint part Rj = Rc (1 + 4K) + 4K (Sm + 1) and a box part
//   B_o = w_o (1 + 4K) + 4K M_o,
// each raised by 1e-6 relative to cover their roundings, so the test stays
// at least as wide as the unsplit one. B_o replaces obs[o].w (every thread
// calls it after box_spheres and a block barrier).
__device__ __forceinline__ void box_limits(const SceneSmem& sc, float4* obs) {
    for (int o = threadIdx.x; o < sc.n_obbs; o += blockDim.x) {
        float4 ob = obs[o];
        const float M = fmaxf(fabsf(ob.x), fmaxf(fabsf(ob.y), fabsf(ob.z)));
        ob.w = (ob.w * (1.0f + 4.0f * PS_GUARD_K) + 4.0f * PS_GUARD_K * M) * (1.0f + 1.0e-6f);
        obs[o] = ob;
    }
}


// Shared-memory view of the staged model core.
struct ModelSmem {
    const BlobHeader* H;
    const JointRec* J;      // full chain, DFS order
    const JointRec* JA;     // approx chain (== J when shared)
    const float4* S;        // exact spheres, reordered
    const int* SO;          // reordered -> descriptor index
    const float4* A;        // approx spheres, reordered
    const int* AO;
};

__device__ __forceinline__ ModelSmem model_view(const unsigned char* blob) {
    ModelSmem m;
    m.H = reinterpret_cast<const BlobHeader*>(blob);
    m.J = reinterpret_cast<const JointRec*>(blob + m.H->off_joints);
    m.JA = m.H->approx_shares_chain ? m.J : reinterpret_cast<const JointRec*>(blob + m.H->off_apx_joints);
    m.S = reinterpret_cast<const float4*>(blob + m.H->off_spheres);
    m.SO = reinterpret_cast<const int*>(blob + m.H->off_sph_orig);
    m.A = reinterpret_cast<const float4*>(blob + m.H->off_apx);
    m.AO = reinterpret_cast<const int*>(blob + m.H->off_apx_orig);
    return m;
}

// Any box hit for one sphere with bit-exact decisions. `cand`/`ncand`
// optionally restrict the boxes (a conservative broad phase); acm_row is the
// sphere's row of an OBB ACM mask (global memory) or NULL.
__device__ __forceinline__ bool sphere_obb_any(const SceneSmem& sc, const uint16_t* cand, int ncand, float px,
                                               float py, float pz, float sr, const uint8_t* acm_row,
                                               LaneStats& st) {
    float lo, hi;
    guard_thresholds(px, py, pz, sr, sc.Bmax, lo, hi);
    const int n = cand ? ncand : sc.n_obbs;
    float mn = 3.0e38f;
    for (int k = 0; k < n; ++k) {
        const int o = cand ? (int)cand[k] : k;
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        mn = fminf(mn, d);
    }
    st.v[ST_PAIRS] += n;
    if (mn < lo) return true;
    if (mn >= hi) return false;
    // Some box sits inside the guard band: re-decide those exactly.
    for (int k = 0; k < n; ++k) {
        const int o = cand ? (int)cand[k] : k;
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        if (d < lo) return true;
        if (d < hi) {
            st.v[ST_EXACT] += 1;
            if (ref_obb_hit(sc.obbs[o], px, py, pz, sr)) return true;
        }
    }
    return false;
}

// Min over boxes of the box SDF of a point (world), no radius. The square
// root and the inside term are taken once per sphere, not per pair:
// SDF = sqrt(min outside d^2) when the centre is outside every box, else the
// most negative max(q) over the boxes that contain it. Also returns min d^2.
__device__ __forceinline__ float sphere_obb_min_sdf(const SceneSmem& sc, float px, float py, float pz,
                                                    const uint8_t* acm_row, float& min_dsq, bool& any_box,
                                                    LaneStats& st) {
    float mn = 3.0e38f;
    any_box = false;
    for (int o = 0; o < sc.n_obbs; ++o) {
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        mn = fminf(mn, fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz));
        any_box = true;
    }
    st.v[ST_PAIRS] += sc.n_obbs;
    min_dsq = mn;
    if (!any_box) return 1000.0f;
    if (mn > 0.0f) return sqrtf(mn);
    float inside = 0.0f;
    for (int o = 0; o < sc.n_obbs; ++o) {
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        if (d == 0.0f) inside = fminf(inside, fmaxf(qx, fmaxf(qy, qz)));
    }
    return inside;
}

// Min d^2 over every box for kN sphere centres at once (one box load per kN
// pair tests); no ACM masks.
template <int kN>
__device__ __forceinline__ void spheres_min_dsq(const SceneSmem& sc, const float* px, const float* py,
                                                const float* pz, float* mn) {
#pragma unroll
    for (int i = 0; i < kN; ++i) mn[i] = 3.0e38f;
    for (int o = 0; o < sc.n_obbs; ++o) {
        const ObbPrep& b = sc.obbs[o];
        const float4 r0 = b.r0, r1 = b.r1, r2 = b.r2, h = b.h;
#pragma unroll
        for (int i = 0; i < kN; ++i) {
            const float lx = fmaf(r0.z, pz[i], fmaf(r0.y, py[i], fmaf(r0.x, px[i], r0.w)));
            const float ly = fmaf(r1.z, pz[i], fmaf(r1.y, py[i], fmaf(r1.x, px[i], r1.w)));
            const float lz = fmaf(r2.z, pz[i], fmaf(r2.y, py[i], fmaf(r2.x, px[i], r2.w)));
            const float cx = fmaxf(fabsf(lx) - h.x, 0.0f), cy = fmaxf(fabsf(ly) - h.y, 0.0f),
                        cz = fmaxf(fabsf(lz) - h.z, 0.0f);
            mn[i] = fminf(mn[i], fmaf(cz, cz, fmaf(cy, cy, cx * cx)));
        }
    }
}

// Packed two-lane FP32 arithmetic of sm_100 (fma/mul .f32x2): each half is
// the IEEE-rounded scalar operation, so a packed chain gives the scalar
// chain's bits; one instruction does the work of two.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Two boxes side by side for the packed loop: every coefficient of box 2k
// in the low half and of box 2k + 1 in the high half (rows of the map with
// the translation, exact half extents). A missing second box is a far one.
struct ObbPair {             // 128 bytes
    f32x2 r0[4], r1[4], r2[4];
    f32x2 h[3];
    f32x2 pad;
};

// Builds the pair table from the staged boxes (every thread calls it; the
// caller syncs after).
__device__ __forceinline__ void stage_obb_pairs(const SceneSmem& sc, ObbPair* pairs) {
    const int np = (sc.n_obbs + 1) / 2;
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
        const ObbPrep& a = sc.obbs[2 * k];
        // a missing second box: identity rows with a 1e15 m translation,
        // d^2 ~ 1e30, never the minimum when a real box exists
        const bool has_b = 2 * k + 1 < sc.n_obbs;
        const ObbPrep& b = sc.obbs[has_b ? 2 * k + 1 : 2 * k];
        const float4 b0 = has_b ? b.r0 : make_float4(1.0f, 0.0f, 0.0f, 1.0e15f);
        const float4 b1 = has_b ? b.r1 : make_float4(0.0f, 1.0f, 0.0f, 1.0e15f);
        const float4 b2 = has_b ? b.r2 : make_float4(0.0f, 0.0f, 1.0f, 1.0e15f);
        const float4 bh = has_b ? b.h : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ObbPair& p = pairs[k];
        p.r0[0] = f2_pack(a.r0.x, b0.x); p.r0[1] = f2_pack(a.r0.y, b0.y);
        p.r0[2] = f2_pack(a.r0.z, b0.z); p.r0[3] = f2_pack(a.r0.w, b0.w);
        p.r1[0] = f2_pack(a.r1.x, b1.x); p.r1[1] = f2_pack(a.r1.y, b1.y);
        p.r1[2] = f2_pack(a.r1.z, b1.z); p.r1[3] = f2_pack(a.r1.w, b1.w);
        p.r2[0] = f2_pack(a.r2.x, b2.x); p.r2[1] = f2_pack(a.r2.y, b2.y);
        p.r2[2] = f2_pack(a.r2.z, b2.z); p.r2[3] = f2_pack(a.r2.w, b2.w);
        p.h[0] = f2_pack(a.h.x, bh.x); p.h[1] = f2_pack(a.h.y, bh.y); p.h[2] = f2_pack(a.h.z, bh.z);
        p.pad = 0ull;
    }
}

// spheres_min_dsq over the pair table: the box map and the squared distance
// of two boxes per packed instruction, each half with fast_box_dsq's
// operation order, so min d^2 has the same bits (min is exact and its order
// does not matter).
template <int kN>
__device__ __forceinline__ void spheres_min_dsq_pairs(const ObbPair* pairs, int n_pairs, const float* px,
                                                      const float* py, const float* pz, float* mn) {
    f32x2 X[kN], Y[kN], Z[kN];
#pragma unroll
    for (int i = 0; i < kN; ++i) {
        mn[i] = 3.0e38f;
        X[i] = f2_pack(px[i], px[i]);
        Y[i] = f2_pack(py[i], py[i]);
        Z[i] = f2_pack(pz[i], pz[i]);
    }
    for (int k = 0; k < n_pairs; ++k) {
        const ObbPair& p = pairs[k];
        const f32x2 a0 = p.r0[0], a1 = p.r0[1], a2 = p.r0[2], a3 = p.r0[3];
        const f32x2 b0 = p.r1[0], b1 = p.r1[1], b2 = p.r1[2], b3 = p.r1[3];
        const f32x2 c0 = p.r2[0], c1 = p.r2[1], c2 = p.r2[2], c3 = p.r2[3];
        float hxa, hxb, hya, hyb, hza, hzb;
        f2_unpack(p.h[0], hxa, hxb);
        f2_unpack(p.h[1], hya, hyb);
        f2_unpack(p.h[2], hza, hzb);
#pragma unroll
        for (int i = 0; i < kN; ++i) {
            const f32x2 lx = f2_fma(a2, Z[i], f2_fma(a1, Y[i], f2_fma(a0, X[i], a3)));
            const f32x2 ly = f2_fma(b2, Z[i], f2_fma(b1, Y[i], f2_fma(b0, X[i], b3)));
            const f32x2 lz = f2_fma(c2, Z[i], f2_fma(c1, Y[i], f2_fma(c0, X[i], c3)));
            float lxa, lxb, lya, lyb, lza, lzb;
            f2_unpack(lx, lxa, lxb);
            f2_unpack(ly, lya, lyb);
            f2_unpack(lz, lza, lzb);
            const f32x2 cx = f2_pack(fmaxf(fabsf(lxa) - hxa, 0.0f), fmaxf(fabsf(lxb) - hxb, 0.0f));
            const f32x2 cy = f2_pack(fmaxf(fabsf(lya) - hya, 0.0f), fmaxf(fabsf(lyb) - hyb, 0.0f));
            const f32x2 cz = f2_pack(fmaxf(fabsf(lza) - hza, 0.0f), fmaxf(fabsf(lzb) - hzb, 0.0f));
            const f32x2 d = f2_fma(cz, cz, f2_fma(cy, cy, f2_mul(cx, cx)));
            float da, db;
            f2_unpack(d, da, db);
            mn[i] = fminf(mn[i], fminf(da, db));
        }
    }
}

// Decision from a precomputed min d^2 (clearance path): exact rescan only
// inside the guard band.
__device__ __forceinline__ bool decide_from_min(const SceneSmem& sc, float px, float py, float pz, float sr,
                                                float min_dsq, const uint8_t* acm_row, LaneStats& st) {
    float lo, hi;
    guard_thresholds(px, py, pz, sr, sc.Bmax, lo, hi);
    if (min_dsq < lo) return true;
    if (min_dsq >= hi) return false;
    for (int o = 0; o < sc.n_obbs; ++o) {
        if (acm_row && acm_row[sc.obb_orig[o]] == 0) continue;
        float qx, qy, qz;
        float d = fast_box_dsq(sc.obbs[o], px, py, pz, qx, qy, qz);
        if (d < lo) return true;
        if (d < hi) {
            st.v[ST_EXACT] += 1;
            if (ref_obb_hit(sc.obbs[o], px, py, pz, sr)) return true;
        }
    }
    return false;
}

// ESDF any-collision / clearance for one sphere over all layers
// (scene_collision.cuh:202-331). acm: sphere_acm_mask row or NULL.
__device__ __forceinline__ bool sphere_esdf_any(const SceneSmem& sc, const ps_scene_view& sv, float px, float py,
                                                float pz, float sr, const uint8_t* acm_row, LaneStats& st) {
    for (int l = 0; l < sc.n_layers; ++l) {
        if (acm_row && acm_row[l] == 0) continue;
        float d;
        st.v[ST_ESDF] += 1;
        if (!esdf_sample(sc.layers[l], sv.voxel_features + (size_t)l * sv.max_voxels_per_layer,
                         sv.max_voxels_per_layer, px, py, pz, sv.esdf_mode, d))
            continue;
        if (d > -sr) return true;
    }
    return false;
}

__device__ __forceinline__ float sphere_esdf_clearance(const SceneSmem& sc, const ps_scene_view& sv, float px,
                                                       float py, float pz, float sr, const uint8_t* acm_row,
                                                       LaneStats& st) {
    float best = 1000.0f;
    for (int l = 0; l < sc.n_layers; ++l) {
        if (acm_row && acm_row[l] == 0) continue;
        float d;
        st.v[ST_ESDF] += 1;
        if (!esdf_sample(sc.layers[l], sv.voxel_features + (size_t)l * sv.max_voxels_per_layer,
                         sv.max_voxels_per_layer, px, py, pz, sv.esdf_mode, d))
            continue;
        best = fminf(best, __fadd_rn(-d, -sr));
    }
    return best;
}

// Select a slot by uniform index.
__device__ __forceinline__ void select_slot(const Affine& s0, const Affine& s1, int k, Affine& out) {
#pragma unroll
    for (int i = 0; i < 12; ++i) out.m[i] = k ? s1.m[i] : s0.m[i];
}

__device__ __forceinline__ void store_slot(Affine& s0, Affine& s1, int k, const Affine& v) {
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        if (k) s1.m[i] = v.m[i];
        else s0.m[i] = v.m[i];
    }
}

// Frame of DFS position p given the parent slots (the reference FK walk).
template <bool kFast>
__device__ __forceinline__ void fk_step(const JointRec& jr, int p, const float* q, Affine& s0, Affine& s1,
                                        Affine& T) {
    if (p == 0) {
        // Both slots start as the identity (runtime_kinematics.cuh:31-37);
        // the first visited joint keeps it.
        affine_identity(T);
    } else {
        Affine P;
        select_slot(s0, s1, jr.parent_slot, P);
        const float qi = jr.dof >= 0 ? q[jr.dof] : 0.0f;
        joint_compose<kFast>(jr, qi, P, T);
    }
    store_slot(s0, s1, jr.slot, T);
}

// ---------------------------------------------------------------------------
// Two-phase self check of one configuration (two_phase_cc.cuh:108-131,
// runtime_kinematics.cuh:249-284 and 383-417): the approximate sphere pairs
// first; the exact pairs only when an approximate pair overlaps; the
// collision margin does not apply to self pairs. Positions of every exact and
// approximate sphere and every joint's bound centre are staged in shared
// memory, SoA by configuration slot (stride kLanes). lane_self_hit checks a
// configuration on one thread (the edge self pass); group_self_hit on a
// group of kSelfSub lanes (the configuration batch).
//
// The exact pairs run by joint pair (a, q), then as the model's runs (sphere
// i of a against the spheres of q): a joint pair is skipped when
// |c_a - c_q| >= R_a + R_q and a run when |p_i - c_q| >= r_i + R_q, each plus
// the guard band, R_q bounding |p_j - c_q| + r_j for every sphere j of q, so
// no pair they hold can pass the float test; the others are tested pair by
// pair with the reference's float test. The verdict is an OR over pairs, so
// the order and the skipped runs change the work, not the result.
// ---------------------------------------------------------------------------
constexpr int kSelfThreads = 64;

// Bound centres are staged only when some joint's cannot be read off its
// first approximate sphere (ModelDev::bound_from_apx); that saves 3 floats per
// joint and slot, which on the Panda lets a fourth self-check block fit on an SM.
struct SelfSmem {
    float *pos, *apos, *cpos;   // [n_spheres*3][L], [n_approx*3][L], [n_joints*3][L] (or none)
    float* end;                 // first float after them
};

template <int kLanes>
__device__ __forceinline__ SelfSmem carve_self(unsigned char* base, int NS, int NA, int NJ, bool bound_from_apx) {
    SelfSmem s;
    s.pos = reinterpret_cast<float*>(base);
    s.apos = s.pos + (size_t)NS * 3 * kLanes;
    s.cpos = s.apos + (size_t)NA * 3 * kLanes;
    s.end = s.cpos + (bound_from_apx ? 0 : (size_t)NJ * 3 * kLanes);
    return s;
}

__device__ __forceinline__ void put3(float* a, int k, int L, int lane, float x, float y, float z) {
    a[(k * 3 + 0) * L + lane] = x;
    a[(k * 3 + 1) * L + lane] = y;
    a[(k * 3 + 2) * L + lane] = z;
}

// The one-thread check of the edge self pass stages each joint's frame (12
// floats) instead of each exact sphere's position (3 floats per sphere: 177
// on the Panda against 96), and transforms a sphere where a joint pair that
// passes its bound test needs it, with the frame it would have been staged
// from, so the positions and the verdict are the same bits. Less shared
// memory per sample lets more samples run per SM.
struct SelfFrames {
    float *fr, *apos, *cpos;   // [n_joints*12][L], [n_approx*3][L], [n_joints*3][L] (or none)
    float* end;                // first float after them
};

template <int kLanes>
__device__ __forceinline__ SelfFrames carve_self_frames(unsigned char* base, int NA, int NJ, bool bound_from_apx) {
    SelfFrames s;
    s.fr = reinterpret_cast<float*>(base);
    s.apos = s.fr + (size_t)NJ * 12 * kLanes;
    s.cpos = s.apos + (size_t)NA * 3 * kLanes;
    s.end = s.cpos + (bound_from_apx ? 0 : (size_t)NJ * 3 * kLanes);
    return s;
}

template <int kLanes>
__device__ bool lane_self_hit(const ModelSmem& M, const ModelDev& md, const float* qc, const SelfFrames& sm, int lane,
                              LaneStats& st) {
    const int NJ = M.H->n_joints;
    float* fr = sm.fr;
    float* apos = sm.apos;
    float* cpos = sm.cpos;
    Affine s0, s1, T;
    affine_identity(s0);
    affine_identity(s1);
    for (int p = 0; p < NJ; ++p) {
        const JointRec& jr = M.J[p];
        fk_step<true>(jr, p, qc, s0, s1, T);
#pragma unroll
        for (int k = 0; k < 12; ++k) fr[(p * 12 + k) * kLanes + lane] = T.m[k];
        if (jr.bound.w >= 0.0f && !md.bound_from_apx) {
            float px, py, pz;
            sphere_world(T, jr.bound.x, jr.bound.y, jr.bound.z, px, py, pz);
            put3(cpos, p, kLanes, lane, px, py, pz);
        }
        if (M.H->approx_shares_chain) {
            for (int k = jr.apx_beg; k < jr.apx_end; ++k) {
                const float4 s = M.A[k];
                float px, py, pz;
                sphere_world(T, s.x, s.y, s.z, px, py, pz);
                put3(apos, k, kLanes, lane, px, py, pz);
            }
        }
    }
    if (!M.H->approx_shares_chain) {
        affine_identity(s0);
        affine_identity(s1);
        for (int p = 0; p < NJ; ++p) {
            const JointRec& jr = M.JA[p];
            fk_step<true>(jr, p, qc, s0, s1, T);
            for (int k = jr.apx_beg; k < jr.apx_end; ++k) {
                const float4 s = M.A[k];
                float px, py, pz;
                sphere_world(T, s.x, s.y, s.z, px, py, pz);
                put3(apos, k, kLanes, lane, px, py, pz);
            }
        }
    }
    auto at = [&](const float* a, int k, int c) { return a[(k * 3 + c) * kLanes + lane]; };
    // a joint's world bound centre (its first approximate sphere's when the model says so)
    auto bc = [&](int p, int c) { return md.bound_from_apx ? at(apos, M.J[p].apx_beg, c) : at(cpos, p, c); };
    auto frame = [&](int p, Affine& F) {
#pragma unroll
        for (int k = 0; k < 12; ++k) F.m[k] = fr[(p * 12 + k) * kLanes + lane];
    };
    bool need = false;
    for (int k = 0; k < M.H->n_apx_self_pairs && !need; ++k) {
        const uint32_t pr = __ldg(md.apx_self_pairs + k);
        const int i = pr & 0xffff, j = pr >> 16;
        st.v[ST_SELF] += 1;
        need = ref_self_hit(at(apos, i, 0), at(apos, i, 1), at(apos, i, 2), M.A[i].w, at(apos, j, 0), at(apos, j, 1),
                            at(apos, j, 2), M.A[j].w);
    }
    if (!need) return false;
    // joint pairs (a, q), nearest in DFS order first: a pair whose bound
    // spheres are apart (|c_a - c_q| >= R_a + R_q plus the guard band) holds
    // no pair that can pass the float test, so its runs are skipped
    for (int jp = 0; jp < md.n_sjp; ++jp) {
        const uint4 e = __ldg(md.sjp + jp);
        const int a = (int)(e.x & 0xffffu), qj = (int)(e.x >> 16);
        {
            const float ax = bc(a, 0), ay = bc(a, 1), az = bc(a, 2);
            const float bx = bc(qj, 0), by = bc(qj, 1), bz = bc(qj, 2);
            const float dx = ax - bx, dy = ay - by, dz = az - bz;
            const float S = fmaxf(fmaxf(fabsf(ax), fmaxf(fabsf(ay), fabsf(az))),
                                  fmaxf(fabsf(bx), fmaxf(fabsf(by), fabsf(bz))));
            float lim = M.J[a].bound.w + M.J[qj].bound.w;
            lim += 4.0f * (S + lim + 1.0f) * PS_GUARD_K;
            st.v[ST_SELF] += 1;
            if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) >= lim * lim * (1.0f + 1.0e-6f)) continue;
        }
        Affine Ta, Tq;
        frame(a, Ta);
        frame(qj, Tq);
        const float4 bq = M.J[qj].bound;
        const float cx = bc(qj, 0), cy = bc(qj, 1), cz = bc(qj, 2);
        for (int r = (int)e.y; r < (int)e.z; ++r) {
            const uint2 run = __ldg(md.sruns + r);
            const int i = run.x & 0x1ff, len = run.x >> 14;
            const float4 si = M.S[i];
            float px, py, pz;
            sphere_world(Ta, si.x, si.y, si.z, px, py, pz);
            const float ri = si.w;
            const float dx = px - cx, dy = py - cy, dz = pz - cz;
            const float S = fmaxf(fmaxf(fabsf(px), fmaxf(fabsf(py), fabsf(pz))), fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz))));
            float lim = ri + bq.w;
            lim += 4.0f * (S + lim + 1.0f) * PS_GUARD_K;
            st.v[ST_SELF] += 1;
            if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) >= lim * lim * (1.0f + 1.0e-6f)) continue;   // no pair can hit
            for (int k = 0; k < len; ++k) {
                const int j = (int)run.y + k;
                const float4 sj = M.S[j];
                float qx, qy, qz;
                sphere_world(Tq, sj.x, sj.y, sj.z, qx, qy, qz);
                st.v[ST_SELF] += 1;
                if (ref_self_hit(px, py, pz, ri, qx, qy, qz, sj.w)) return true;
            }
        }
    }
    return false;
}

// kSelfSub consecutive lanes check one configuration (a group; slot = the
// configuration's column in the staged positions, u = the lane within the
// group). Every lane of the group walks the FK and stores its share of the
// sphere positions (spheres u, u + kSelfSub, ... of each joint); the group's
// lanes then split the approximate pairs and, per joint pair that passes its
// bound test, the runs, each lane to its own first hit, with one group ballot
// per phase (the verdict is an OR, so the split changes the work, not the
// result). The check of a few
// thousand configurations is latency-bound: one lane per configuration left
// 3 warps per SM for the same shared memory (16,384 CHOMP waypoints: 49.6 ->
// 26.5 us with a ballot after every round, 24.0 us with one per phase). The edge self pass keeps lane_self_hit: its windows of samples
// ran slower with groups of 2 or 4 lanes (107 -> 135 and 124 us).
constexpr int kSelfSub = 4;
constexpr int kSelfBlock = kSelfThreads * kSelfSub;   // threads of a self-check block

template <int kSlots>
__device__ bool group_self_hit(const ModelSmem& M, const ModelDev& md, const float* qc, const SelfSmem& sm, int slot,
                               int u, LaneStats& st) {
    const int NJ = M.H->n_joints;
    const unsigned gmask = 0xfu << ((threadIdx.x & 31) & ~(kSelfSub - 1));
    float* pos = sm.pos;
    float* apos = sm.apos;
    float* cpos = sm.cpos;
    Affine s0, s1, T;
    affine_identity(s0);
    affine_identity(s1);
    for (int p = 0; p < NJ; ++p) {
        const JointRec& jr = M.J[p];
        fk_step<true>(jr, p, qc, s0, s1, T);
        for (int k = jr.sph_beg + u; k < jr.sph_end; k += kSelfSub) {
            const float4 s = M.S[k];
            float px, py, pz;
            sphere_world(T, s.x, s.y, s.z, px, py, pz);
            put3(pos, k, kSlots, slot, px, py, pz);
        }
        if (u == 0 && jr.bound.w >= 0.0f && !md.bound_from_apx) {
            float px, py, pz;
            sphere_world(T, jr.bound.x, jr.bound.y, jr.bound.z, px, py, pz);
            put3(cpos, p, kSlots, slot, px, py, pz);
        }
        if (M.H->approx_shares_chain) {
            for (int k = jr.apx_beg + u; k < jr.apx_end; k += kSelfSub) {
                const float4 s = M.A[k];
                float px, py, pz;
                sphere_world(T, s.x, s.y, s.z, px, py, pz);
                put3(apos, k, kSlots, slot, px, py, pz);
            }
        }
    }
    if (!M.H->approx_shares_chain) {
        affine_identity(s0);
        affine_identity(s1);
        for (int p = 0; p < NJ; ++p) {
            const JointRec& jr = M.JA[p];
            fk_step<true>(jr, p, qc, s0, s1, T);
            for (int k = jr.apx_beg + u; k < jr.apx_end; k += kSelfSub) {
                const float4 s = M.A[k];
                float px, py, pz;
                sphere_world(T, s.x, s.y, s.z, px, py, pz);
                put3(apos, k, kSlots, slot, px, py, pz);
            }
        }
    }
    __syncwarp(gmask);   // the group's positions are written
    auto at = [&](const float* a, int k, int c) { return a[(k * 3 + c) * kSlots + slot]; };
    // a joint's world bound centre (its first approximate sphere's when the model says so)
    auto bc = [&](int p, int c) { return md.bound_from_apx ? at(apos, M.J[p].apx_beg, c) : at(cpos, p, c); };
    // each lane runs its share to its own first hit; the group ballots once
    // per phase (the verdict is an OR, so a lane's early stop changes nothing)
    bool need = false;
    for (int k = u; k < M.H->n_apx_self_pairs && !need; k += kSelfSub) {
        const uint32_t pr = __ldg(md.apx_self_pairs + k);
        const int i = pr & 0xffff, j = pr >> 16;
        st.v[ST_SELF] += 1;
        need = ref_self_hit(at(apos, i, 0), at(apos, i, 1), at(apos, i, 2), M.A[i].w, at(apos, j, 0), at(apos, j, 1),
                            at(apos, j, 2), M.A[j].w);
    }
    if (!__ballot_sync(gmask, need)) return false;
    bool hit = false;
    // joint pairs (a, q), nearest in DFS order first: a pair whose bound
    // spheres are apart (|c_a - c_q| >= R_a + R_q plus the guard band) holds
    // no pair that can pass the float test, so its runs are skipped
    for (int jp = 0; jp < md.n_sjp && !hit; ++jp) {
        const uint4 e = __ldg(md.sjp + jp);
        const int a = (int)(e.x & 0xffffu), qj = (int)(e.x >> 16);
        {
            const float ax = bc(a, 0), ay = bc(a, 1), az = bc(a, 2);
            const float bx = bc(qj, 0), by = bc(qj, 1), bz = bc(qj, 2);
            const float dx = ax - bx, dy = ay - by, dz = az - bz;
            const float S = fmaxf(fmaxf(fabsf(ax), fmaxf(fabsf(ay), fabsf(az))),
                                  fmaxf(fabsf(bx), fmaxf(fabsf(by), fabsf(bz))));
            float lim = M.J[a].bound.w + M.J[qj].bound.w;
            lim += 4.0f * (S + lim + 1.0f) * PS_GUARD_K;
            if (u == 0) st.v[ST_SELF] += 1;
            if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) >= lim * lim * (1.0f + 1.0e-6f)) continue;
        }
        const float4 bq = M.J[qj].bound;
        const float cx = bc(qj, 0), cy = bc(qj, 1), cz = bc(qj, 2);
        for (int r = (int)e.y + u; r < (int)e.z && !hit; r += kSelfSub) {
            const uint2 run = __ldg(md.sruns + r);
            const int i = run.x & 0x1ff, len = run.x >> 14;
            const float px = at(pos, i, 0), py = at(pos, i, 1), pz = at(pos, i, 2), ri = M.S[i].w;
            const float dx = px - cx, dy = py - cy, dz = pz - cz;
            const float S = fmaxf(fmaxf(fabsf(px), fmaxf(fabsf(py), fabsf(pz))),
                                  fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz))));
            float lim = ri + bq.w;
            lim += 4.0f * (S + lim + 1.0f) * PS_GUARD_K;
            st.v[ST_SELF] += 1;
            if (fmaf(dz, dz, fmaf(dy, dy, dx * dx)) >= lim * lim * (1.0f + 1.0e-6f)) continue;   // no pair can hit
            for (int k = 0; k < len && !hit; ++k) {
                const int j = (int)run.y + k;
                st.v[ST_SELF] += 1;
                hit = ref_self_hit(px, py, pz, ri, at(pos, j, 0), at(pos, j, 1), at(pos, j, 2), M.S[j].w);
            }
        }
    }
    return __ballot_sync(gmask, hit) != 0;
}

// Shared memory of a self-check block (kSelfThreads configuration slots): model
// core, sphere and bound positions and a tile of configurations.
inline size_t self_smem_bytes(const ps_model* m) {
    const int nc = m->dev.bound_from_apx ? 0 : m->info.n_joints;
    return (size_t)m->dev.bytes_core +
           (size_t)(m->info.n_spheres + m->info.n_approx_spheres + nc) * 3 * kSelfThreads * 4 +
           (size_t)kSelfThreads * m->info.n_dof * 4;
}

// PS_EINVAL with the sizes when the self check's block does not fit in shared
// memory: about 280 spheres, approximate spheres and joints together on a
// B200 (the reference's edge kernel stages at most 125 spheres, 52
// approximate ones: edge_eval.cuh:83-84).
// Shared memory of an edge self-pass block (lane_self_hit, kSelfThreads
// samples): model core, frames, approximate sphere positions, bound centres
// when they are staged, a tile of configurations.
inline size_t self_lane_smem_bytes(const ps_model* m) {
    const int nc = m->dev.bound_from_apx ? 0 : m->info.n_joints;
    return (size_t)m->dev.bytes_core +
           (size_t)(12 * m->info.n_joints + 3 * m->info.n_approx_spheres + 3 * nc) * kSelfThreads * 4 +
           (size_t)kSelfThreads * m->info.n_dof * 4;
}

inline int check_self_fits(const ps_model* m) {
    const size_t need = self_smem_bytes(m), have = smem_optin();
    if (need <= have) return PS_OK;
    return set_error(PS_EINVAL, "check_self: n_spheres + n_approx_spheres + n_joints = " +
                                    std::to_string(m->info.n_spheres + m->info.n_approx_spheres + m->info.n_joints) +
                                    " needs " + std::to_string(need) + " bytes of shared memory per block, above the "
                                    "device's " + std::to_string(have));
}

}  // namespace ps
