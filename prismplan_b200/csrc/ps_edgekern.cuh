// ps_edgekern.cuh -- edge-check kernels shared by the edge entry points
// (ps_edges.cu) and the mixed-request batch (ps_batch.cu). Each translation
// unit that includes this header gets its own private copy of the kernels.
#pragma once

#include <algorithm>
#include <cfloat>

#include "ps_internal.h"
#include "ps_verdict.cuh"

namespace ps {

namespace {

constexpr int kWarps = 4;               // warps per block
constexpr int kEdgeThreads = 32 * kWarps;
constexpr unsigned kFull = 0xffffffffu;

struct EdgeWs {                         // header of the persistent workspace (64 B)
    unsigned long long head[2];         // next chunk-major item of each pass
    unsigned long long deadline;        // %globaltimer deadline (ns), 0 = none
    unsigned long long self_samples;    // samples of every edge (self pass sizing)
    int max_rounds;                     // most chunk rounds of any edge
    int timed_out;                      // set once a queue kernel stops at the deadline
    int self_edges;                     // edges with at least one sample
    int self_next;                      // next window of the self pass
    int wp_next;                        // next waypoint group (the batch's work-queue kernel)
    int n_long;                         // edges with more than one chunk round (the long list)
    int pad[2];
};
static_assert(sizeof(EdgeWs) == 64, "the workspace header is 64 B");

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Chunk visiting order of an edge with nc chunks of 32 samples: with
// s = ceil(sqrt(nc)) and m = ceil(nc / s), round k visits chunk
// (k % m) * s + k / m, so the first rounds spread over the whole edge and a
// colliding stretch is found, and the edge retired, after fewer chunks than
// in order. Rounds whose chunk is >= nc are empty. The verdict is the OR over
// all samples, so the order changes only the work, never the result.
struct ChunkOrder {
    int nc, s, m;
    __device__ __forceinline__ explicit ChunkOrder(int G) {
        nc = G > 0 ? (G + 31) / 32 : 0;
        s = nc > 0 ? (int)ceilf(sqrtf((float)nc)) : 1;
        while (s > 1 && (s - 1) * (s - 1) >= nc) --s;   // exact integer ceil(sqrt)
        while (s * s < nc) ++s;
        m = nc > 0 ? (nc + s - 1) / s : 0;
    }
    __device__ __forceinline__ int rounds() const { return m * s; }
    __device__ __forceinline__ int chunk(int k) const { return (k % m) * s + k / m; }
};

__device__ __forceinline__ int ordered_float(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : (i ^ 0x7fffffff);
}
__device__ __forceinline__ float unordered_float(int i) { return __int_as_float(i >= 0 ? i : (i ^ 0x7fffffff)); }

// Sample count of an edge (edge_eval.cuh:54-60 plus the L-inf rule).
__device__ __forceinline__ int edge_samples(const ps_edge_params& P, const int* given, int e, const float* a,
                                            const float* b, int D, float len) {
    if (given) return given[e];
    if (P.resolution > 0.0f) {
        int g = (int)ceilf(__fdiv_rn(len, P.resolution));
        return min(max(g, 2), 1024);
    }
    if (P.max_joint_step > 0.0f) {
        float m = 0.0f;
        for (int i = 0; i < D; ++i) m = fmaxf(m, fabsf(__fadd_rn(b[i], -a[i])));
        int g = (int)ceilf(__fdiv_rn(m, P.max_joint_step));
        const int cap = P.max_samples > 0 ? P.max_samples : 1024;
        return min(max(g, 1), cap);
    }
    return P.granularity;
}

__device__ __forceinline__ float edge_length(const float* a, const float* b, int D) {
    float len2 = 0.0f;   // edge_eval.cuh:104-106
    for (int i = 0; i < D; ++i) {
        float d = __fadd_rn(b[i], -a[i]);
        len2 = __fmaf_rn(d, d, len2);
    }
    return sqrtf(len2);
}

struct WarpScratch {
    float* q;          // [32 * D]
    uint16_t* cand;    // [n_obbs]
    const float4* obs; // [n_obbs] box centre, .w its part of the broad-phase limit (block-wide)
};

// One chunk of one edge. Returns true if any sample of the chunk collides.
// Every lane of the warp must call it. clr_min (may be NULL) receives the
// min ESDF clearance over the chunk's samples when compute_clearance.
__device__ bool process_chunk(const ModelSmem& M, const SceneSmem& sc, const ps_scene_view& sv,
                              const ps_edge_params& P, const float* __restrict__ from,
                              const float* __restrict__ to, int e, int G, int chunk, WarpScratch ws,
                              float* clr_min, LaneStats& st_out) {
    const int lane = threadIdx.x & 31;
    LaneStats st;   // padding lanes repeat a sample: their work is not credited
    st.zero();
    const int D = M.H->n_dof, NJ = M.H->n_joints;
    // Reference sampling (edge_eval.cuh:110-121): t = j/G for j = 1..G in
    // slots of 16; slots past G take t = 0, i.e. the start configuration,
    // and their verdict counts. So the start configuration belongs to the
    // edge verdict exactly when G % 16 != 0; a padding lane of the last chunk
    // carries it (such a lane exists whenever G % 16 != 0), the remaining
    // padding lanes repeat sample G and are not counted.
    const int j_raw = chunk * 32 + lane + 1;
    const bool in_range = j_raw <= G;
    const bool start_lane = !in_range && (G % 16) != 0 && j_raw == G + 1;
    const bool real = in_range || start_lane;
    const int j = in_range ? j_raw : (start_lane ? 0 : G);
    const float t = __fdiv_rn((float)j, (float)G);
    const float* a = from + (size_t)e * D;
    const float* b = to + (size_t)e * D;
    float* qc = ws.q + lane * D;
    for (int i = 0; i < D; ++i) {
        const float ai = __ldg(a + i), bi = __ldg(b + i);
        qc[i] = __fmaf_rn(t, __fadd_rn(bi, -ai), ai);
    }
    __syncwarp();
    if (real) st.v[ST_SAMPLES] += 1;
    const float margin = P.collision_margin;
    const bool shares = M.H->approx_shares_chain != 0;
    const bool want_clr = P.compute_clearance != 0 && clr_min != nullptr;

    Affine s0, s1, T, a0, a1, TA;
    affine_identity(s0);
    affine_identity(s1);
    affine_identity(a0);
    affine_identity(a1);
    bool hit = false;
    float clr = 1000.0f;
    for (int p = 0; p < NJ; ++p) {
        const JointRec& jr = M.J[p];
        fk_step<true>(jr, p, qc, s0, s1, T);
        if (!shares) fk_step<true>(M.JA[p], p, qc, a0, a1, TA);
        st.v[ST_JOINTS] += (p > 0 && real);
        const bool has_spheres = jr.sph_end > jr.sph_beg || jr.apx_end > jr.apx_beg;
        if (!has_spheres) continue;   // uniform across the warp

        // ---- warp broad phase over boxes ----
        const uint16_t* cand = nullptr;
        int ncand = sc.n_obbs;
        if (shares && sc.n_obbs > 0 && jr.bound.w >= 0.0f) {
            float cx, cy, cz;
            sphere_world(T, jr.bound.x, jr.bound.y, jr.bound.z, cx, cy, cz);
            float mx = cx, my = cy, mz = cz;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mx += __shfl_xor_sync(kFull, mx, o);
                my += __shfl_xor_sync(kFull, my, o);
                mz += __shfl_xor_sync(kFull, mz, o);
            }
            mx *= (1.0f / 32.0f);
            my *= (1.0f / 32.0f);
            mz *= (1.0f / 32.0f);
            const float dx = cx - mx, dy = cy - my, dz = cz - mz;
            float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r2 = fmaxf(r2, __shfl_xor_sync(kFull, r2, o));
            const float S = fmaxf(fabsf(mx), fmaxf(fabsf(my), fabsf(mz)));
            float Rc = sqrtf(r2) + jr.bound.w + fmaxf(margin, 0.0f);
            Rc += 4.0f * (S + Rc + sc.Bmax + 1.0f) * PS_GUARD_K;
            const float Rcl = Rc * sc.Mscale;   // world radius -> box-frame radius (map stretch)
        const float Rc2 = Rcl * Rcl;
            int count = 0;
            __syncwarp();   // previous joint's readers of ws.cand are done
            for (int base = 0; base < sc.n_obbs; base += 32) {
                const int o = base + lane;
                bool keep = false;
                if (o < sc.n_obbs) {
                    float qx, qy, qz;
                    keep = fast_box_dsq(sc.obbs[o], mx, my, mz, qx, qy, qz) < Rc2;
                    st.v[ST_CULL] += 1;
                }
                const unsigned bal = __ballot_sync(kFull, keep);
                if (keep) ws.cand[count + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)o;
                count += __popc(bal);
            }
            __syncwarp();
            cand = ws.cand;
            ncand = count;
            if (count == 0 && sc.n_layers == 0 && !want_clr) continue;   // nothing reachable
        }

        // ---- approximate gate ----
        bool flagged = false;
        for (int k = jr.apx_beg; k < jr.apx_end && !flagged; ++k) {
            const float4 sa = M.A[k];
            float px, py, pz;
            sphere_world(shares ? T : TA, sa.x, sa.y, sa.z, px, py, pz);
            if (real) st.v[ST_SPHERES] += 1;
            const float sr = __fadd_rn(sa.w, margin);
            // no mask in the approximate pass (sphere index -1 in the
            // reference, scene_collision.cuh:584-606)
            flagged = (ncand > 0 && sphere_obb_any(sc, cand, ncand, px, py, pz, sr, nullptr, st)) ||
                      (sc.n_layers && sphere_esdf_any(sc, sv, px, py, pz, sr, nullptr, st));
        }
        // ---- exact spheres of a flagged joint (and ESDF clearance) ----
        const bool decide = flagged && !hit;
        if (decide || want_clr) {
            for (int k = jr.sph_beg; k < jr.sph_end; ++k) {
                const float4 sp = M.S[k];
                float px, py, pz;
                sphere_world(T, sp.x, sp.y, sp.z, px, py, pz);
                if (real) st.v[ST_SPHERES] += 1;
                const float sr = __fadd_rn(sp.w, margin);
                const int so = M.SO[k];
                const uint8_t* eacm =
                    sv.sphere_acm_mask ? sv.sphere_acm_mask + (size_t)so * sv.n_voxel_layers : nullptr;
                if (want_clr && sc.n_layers) clr = fminf(clr, sphere_esdf_clearance(sc, sv, px, py, pz, sr, eacm, st));
                if (decide && !hit) {
                    const uint8_t* acm =
                        sv.sphere_obb_acm_mask ? sv.sphere_obb_acm_mask + (size_t)so * sv.n_obbs : nullptr;
                    hit = (ncand > 0 && sphere_obb_any(sc, cand, ncand, px, py, pz, sr, acm, st)) ||
                          (sc.n_layers && sphere_esdf_any(sc, sv, px, py, pz, sr, eacm, st));
                    if (hit && !want_clr) break;
                }
            }
        }
        if (!want_clr && __any_sync(kFull, hit && real)) break;   // warp-uniform early exit
    }
    if (want_clr) {
        float c = in_range ? clr : 3.0e38f;   // clearance covers j = 1..G only (edge_eval.cuh:146-151)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c = fminf(c, __shfl_xor_sync(kFull, c, o));
        *clr_min = c;
    }
    if (real)
        for (int k = 0; k < ST_COUNT; ++k) st_out.v[k] += st.v[k];
    return __any_sync(kFull, hit && real);
}

// Fast path of process_chunk for the common scene: the approximate chain is
// the full chain, no ACM masks, no ESDF layers, no clearance. Same verdict;
// fewer live registers and a per-joint guard band. Exact spheres are tested 4
// at a time (2 with ESDF layers) against each surviving box (one box load per
// group), then decided from their min d^2 with the exact re-decision inside
// the guard band.
//
// Code size matters here: the kernel issues about 3 of every 4 cycles, and
// instruction fetch stalls were the third largest stall reason. The box loops
// are kept rolled and the rare band re-decision is out of line, which took
// 7 % (boxes only) and 15 % (boxes and ESDF) off the kernel time.

// Exact re-decision of one sphere whose min d^2 fell inside the guard band
// (lo, hi): the band's boxes are decided one by one with the reference test.
__device__ __noinline__ bool band_redecide(const SceneSmem& sc, const uint16_t* cand, int ncand, float px, float py,
                                           float pz, float sr, float lo, float hi, LaneStats& st) {
    for (int k = 0; k < ncand; ++k) {
        const ObbPrep& o = sc.obbs[cand[k]];
        float qx, qy, qz;
        const float d = fast_box_dsq(o, px, py, pz, qx, qy, qz);
        if (d < lo) return true;
        if (d < hi) {
            st.v[ST_EXACT] += 1;
            if (ref_obb_hit(o, px, py, pz, sr)) return true;
        }
    }
    return false;
}

// Decide one sphere from its min d^2 over the candidate boxes: definite
// outside the guard band, exact re-decision of the band's boxes otherwise.
__device__ __forceinline__ bool decide_band(const SceneSmem& sc, const uint16_t* cand, int ncand, float px, float py,
                                            float pz, float sr, float g, float mn, LaneStats& st) {
    const float a = fmaxf(sr - g, 0.0f), b = sr + g;
    const float lo = a * a * (1.0f - 1.0e-6f), hi = b * b * (1.0f + 1.0e-6f);
    if (mn < lo) return true;
    if (mn >= hi) return false;
    return band_redecide(sc, cand, ncand, px, py, pz, sr, lo, hi, st);
}

// kN spheres (positions in registers) against every candidate box: one box
// load per kN pair tests. Returns whether any of them hits.
template <int kN, bool kStats>
__device__ __forceinline__ bool spheres_hit(const SceneSmem& sc, const uint16_t* cand, int ncand, const float* px,
                                            const float* py, const float* pz, const float* sr, float g,
                                            LaneStats& st) {
    float mn[kN];
#pragma unroll
    for (int i = 0; i < kN; ++i) mn[i] = 3.0e38f;
#pragma unroll 1
    for (int k = 0; k < ncand; ++k) {
        const ObbPrep& o = sc.obbs[cand[k]];
        const float4 r0 = o.r0, r1 = o.r1, r2 = o.r2, h = o.h;
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
    if (kStats) st.v[ST_PAIRS] += ncand * kN;
    bool hit = false;
#pragma unroll
    for (int i = 0; i < kN; ++i)
        if (!hit) hit = decide_band(sc, cand, ncand, px[i], py[i], pz[i], sr[i], g, mn[i], st);
    return hit;
}

// Approximate gate of one joint for this lane: any approximate sphere hits a
// candidate box (or an ESDF layer).
template <bool kStats, bool kEsdf>
__device__ __forceinline__ bool joint_gate(const ModelSmem& M, const SceneSmem& sc, const ps_scene_view& sv,
                                           const JointRec& jr, const Affine& T, float margin, const WarpScratch& ws,
                                           int ncand, float g, LaneStats& st) {
    bool flagged = false;
    for (int a = jr.apx_beg; a < jr.apx_end && !flagged; ++a) {
        const float4 sa = M.A[a];
        float px, py, pz;
        sphere_world(T, sa.x, sa.y, sa.z, px, py, pz);
        const float sr = __fadd_rn(sa.w, margin);
        if (kStats) st.v[ST_SPHERES] += 1;
        flagged = spheres_hit<1, kStats>(sc, ws.cand, ncand, &px, &py, &pz, &sr, g, st) ||
                  (kEsdf && sphere_esdf_any(sc, sv, px, py, pz, sr, nullptr, st));
    }
    return flagged;
}

template <bool kStats, bool kEsdf>
__device__ bool process_chunk_fast(const ModelSmem& M, const SceneSmem& sc, const ps_scene_view& sv,
                                   const ps_edge_params& P,
                                   const float* __restrict__ from, const float* __restrict__ to, int e, int G,
                                   int chunk, WarpScratch ws, LaneStats& st_out) {
    const int lane = threadIdx.x & 31;
    LaneStats st;
    st.zero();
    const int D = M.H->n_dof, NJ = M.H->n_joints;
    // sampling rule as in process_chunk (edge_eval.cuh:110-121)
    const int j_raw = chunk * 32 + lane + 1;
    const bool in_range = j_raw <= G;
    const bool start_lane = !in_range && (G % 16) != 0 && j_raw == G + 1;
    const bool real = in_range || start_lane;
    const int j = in_range ? j_raw : (start_lane ? 0 : G);
    const float t = __fdiv_rn((float)j, (float)G);
    const float* a = from + (size_t)e * D;
    const float* b = to + (size_t)e * D;
    float* qc = ws.q + lane * D;
    for (int i = 0; i < D; ++i) {
        const float ai = __ldg(a + i), bi = __ldg(b + i);
        qc[i] = __fmaf_rn(t, __fadd_rn(bi, -ai), ai);
    }
    __syncwarp();
    if (kStats && real) st.v[ST_SAMPLES] += 1;
    const float margin = P.collision_margin;
    // Slot 0 holds only the root's identity frame (checked on the host), so a
    // joint's parent frame is the identity or the current frame: one 3x4
    // frame in registers. Composing with the identity reproduces the step
    // exactly, as the reference's slot walk does.
    Affine T;
    affine_identity(T);
    bool hit = false;
    for (int p = 0; p < NJ; ++p) {
        const JointRec& jr = M.J[p];
        if (p > 0) {
            const float qi = jr.dof >= 0 ? qc[jr.dof] : 0.0f;
            if (jr.parent_slot == 0) {
                Affine I;
                affine_identity(I);
                joint_compose<true>(jr, qi, I, T);
            } else {
                joint_compose<true>(jr, qi, T, T);   // rows are read before they are written
            }
            if (kStats) st.v[ST_JOINTS] += 1;
        }
        if (jr.bound.w < 0.0f || (sc.n_obbs == 0 && !kEsdf)) continue;   // nothing to test (uniform)
        // ---- warp broad phase: one sphere around the joint's bound spheres of
        //      all 32 samples, centred on the middle sample's ----
        float cx, cy, cz;
        sphere_world(T, jr.bound.x, jr.bound.y, jr.bound.z, cx, cy, cz);
        const float mx = __shfl_sync(kFull, cx, 16), my = __shfl_sync(kFull, cy, 16),
                    mz = __shfl_sync(kFull, cz, 16);
        const float dx = cx - mx, dy = cy - my, dz = cz - mz;
        // max over lanes in one warp reduction: non-negative floats order as their bits
        const float r2 = __uint_as_float(__reduce_max_sync(kFull, __float_as_uint(fmaf(dz, dz, fmaf(dy, dy, dx * dx)))));
        const float Sm = fmaxf(fabsf(mx), fmaxf(fabsf(my), fabsf(mz)));
        // the square root only widens a conservative bound: the approximate
        // one, raised by 1e-6 relative (far above its error), is enough
        const float r2c = fmaxf(r2, 1.0e-30f);
        float Rc = r2c * rsqrtf(r2c) * (1.0f + 1.0e-6f) + jr.bound.w + fmaxf(margin, 0.0f);
        Rc += 4.0f * (Sm + Rc + sc.Bmax + 1.0f) * PS_GUARD_K;
        const float Rcl = Rc * sc.Mscale;   // world radius -> box-frame radius (map stretch)
        const float Rc2 = Rcl * Rcl;
        const float Rj = (Rc * (1.0f + 4.0f * PS_GUARD_K) + 4.0f * PS_GUARD_K * (Sm + 1.0f)) * (1.0f + 1.0e-6f);
        int ncand = 0;
        __syncwarp();
#pragma unroll 1
        for (int base = 0; base < sc.n_obbs; base += 32) {
            const int o = base + lane;
            bool keep = false;
            if (o < sc.n_obbs) {
                // circumscribed-sphere test first, the box distance only if it passes
                const float4 ob = ws.obs[o];
                const float ex = ob.x - mx, ey = ob.y - my, ez = ob.z - mz;
                const float lim = Rj + ob.w;   // see box_limits
                if (fmaf(ez, ez, fmaf(ey, ey, ex * ex)) < lim * lim) {
                    float qx, qy, qz;
                    keep = fast_box_dsq(sc.obbs[o], mx, my, mz, qx, qy, qz) < Rc2;
                }
                if (kStats) st.v[ST_CULL] += 1;
            }
            const unsigned bal = __ballot_sync(kFull, keep);
            if (keep) ws.cand[ncand + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)o;
            ncand += __popc(bal);
        }
        __syncwarp();
        // ESDF layers within reach of any sphere of the joint over the chunk (uniform)
        const bool esdf = kEsdf && esdf_reachable(sc, mx, my, mz, Rc);
        if (ncand == 0 && !esdf) continue;   // nothing reachable from any lane (uniform)
        // Per-joint guard: every sphere of the joint lies within bound.w of c.
        const float S = fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz))) + jr.bound.w;
        const float g = (S + sc.Bmax + 1.0f) * PS_GUARD_K;
        // ---- the joint's verdict is gate && exact (two_phase_cc.cuh:57-138).
        //      Boxes only: exact spheres first, the approximate gate only for a
        //      lane whose exact spheres hit. With an ESDF layer in reach the
        //      gate comes first, so unflagged joints skip the exact spheres'
        //      ESDF lookups. ----
        if (!hit) {
            bool flagged = false;
            if (esdf) flagged = joint_gate<kStats, true>(M, sc, sv, jr, T, margin, ws, ncand, g, st);
            bool ex = false;
            if (!esdf || flagged) {
                int k = jr.sph_beg;
                // spheres per box load: 4 with boxes only, 2 when the ESDF
                // lookups share the registers (measured best for each)
                constexpr int kG = kEsdf ? 2 : 4;
                for (; k + kG <= jr.sph_end && !ex; k += kG) {
                    float px[kG], py[kG], pz[kG], sr[kG];
#pragma unroll
                    for (int i = 0; i < kG; ++i) {
                        const float4 sp = M.S[k + i];
                        sphere_world(T, sp.x, sp.y, sp.z, px[i], py[i], pz[i]);
                        sr[i] = __fadd_rn(sp.w, margin);
                    }
                    if (kStats) st.v[ST_SPHERES] += kG;
                    ex = spheres_hit<kG, kStats>(sc, ws.cand, ncand, px, py, pz, sr, g, st);
                    if (esdf)
#pragma unroll
                        for (int i = 0; i < kG; ++i)
                            if (!ex) ex = sphere_esdf_any(sc, sv, px[i], py[i], pz[i], sr[i], nullptr, st);
                }
                for (; k < jr.sph_end && !ex; ++k) {
                    const float4 sp = M.S[k];
                    float px, py, pz;
                    sphere_world(T, sp.x, sp.y, sp.z, px, py, pz);
                    const float sr = __fadd_rn(sp.w, margin);
                    if (kStats) st.v[ST_SPHERES] += 1;
                    ex = spheres_hit<1, kStats>(sc, ws.cand, ncand, &px, &py, &pz, &sr, g, st) ||
                         (esdf && sphere_esdf_any(sc, sv, px, py, pz, sr, nullptr, st));
                }
            }
            if (!esdf && ex) flagged = joint_gate<kStats, false>(M, sc, sv, jr, T, margin, ws, ncand, g, st);
            hit = ex && flagged;
        }
        if (__any_sync(kFull, hit && real)) break;   // warp-uniform early exit
    }
    if (kStats && real)
        for (int k = 0; k < ST_COUNT; ++k) st_out.v[k] += st.v[k];
    return __any_sync(kFull, hit && real);
}

// Shared-memory carve-up common to both edge kernels.
struct EdgeSmem {
    unsigned char* blob;
    ObbPrep* obbs;
    int* orig;
    LayerPrep* layers;
    float* q;          // [kWarps][32*D]
    uint16_t* cand;    // [kWarps][n_obbs_pad]
    float4* obs;       // [n_obbs]
};

__device__ __forceinline__ EdgeSmem carve(unsigned char* smem, const ModelDev& md, const ps_scene_view& sv, int D) {
    EdgeSmem s;
    s.blob = smem;
    s.obbs = reinterpret_cast<ObbPrep*>(smem + md.bytes_core);
    const int nob = max(sv.n_obbs, 1);
    s.orig = reinterpret_cast<int*>(s.obbs + nob);
    s.layers = reinterpret_cast<LayerPrep*>(s.orig + ((nob + 3) & ~3));
    s.q = reinterpret_cast<float*>(s.layers + PS_MAX_LAYERS);
    s.cand = reinterpret_cast<uint16_t*>(s.q + kWarps * 32 * D);
    const int nob_pad = (nob + 7) & ~7;
    s.obs = reinterpret_cast<float4*>(s.cand + kWarps * nob_pad);
    return s;
}

size_t edge_smem_bytes(const ps_model* m, const ps_scene_view* sv) {
    const int nob_pad = (std::max(sv->n_obbs, 1) + 7) & ~7;
    return (size_t)m->dev.bytes_core + scene_smem_bytes(sv) + (size_t)kWarps * 32 * m->info.n_dof * 4 +
           (size_t)kWarps * nob_pad * 2 + (size_t)16 * std::max(sv->n_obbs, 1) + 64;
}

// ---------------------------------------------------------------------------
// Plain path: one warp per edge, chunks in order.
// ---------------------------------------------------------------------------
template <int kMode, bool kStats>
__global__ void __launch_bounds__(kEdgeThreads, kMode ? 6 : 3) edges_plain_kernel(ModelDev md, ps_scene_view sv, ps_edge_params P,
                                                                  const float* __restrict__ from,
                                                                  const float* __restrict__ to,
                                                                  const int* __restrict__ given, int n_edges,
                                                                  uint8_t* __restrict__ valid, float* __restrict__ cost,
                                                                  float* __restrict__ clearance,
                                                                  unsigned long long* stats) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (!stage_model(md, smem, &mbar)) {   // fail closed: this block's edges come back invalid
        for (int e = blockIdx.x * kWarps + warp; e < n_edges; e += gridDim.x * kWarps)
            if (lane == 0) {
                valid[e] = 0;
                cost[e] = FLT_MAX;
                if (clearance) clearance[e] = __int_as_float(0x7fc00000);
            }
        return;
    }
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof;
    EdgeSmem es = carve(smem, md, sv, D);
    SceneSmem sc;
    stage_scene(sv, es.obbs, es.orig, es.layers, counters, &bmax, sc);
    box_spheres(sc, es.obs);
    __syncthreads();
    box_limits(sc, es.obs);
    __syncthreads();
    const int nob_pad = (max(sv.n_obbs, 1) + 7) & ~7;
    WarpScratch ws{es.q + warp * 32 * D, es.cand + warp * nob_pad, es.obs};
    LaneStats st;
    st.zero();
    for (int e = blockIdx.x * kWarps + warp; e < n_edges; e += gridDim.x * kWarps) {
        const float* a = from + (size_t)e * D;
        const float* b = to + (size_t)e * D;
        const float len = edge_length(a, b, D);
        const int G = edge_samples(P, given, e, a, b, D, len);
        bool bad = false;
        float emin = FLT_MAX;
        const ChunkOrder ord(G);
        for (int r = 0; r < ord.rounds(); ++r) {
            const int c = ord.chunk(r);
            if (c >= ord.nc) continue;
            float cm = FLT_MAX;
            if (kMode) bad |= process_chunk_fast<kStats, kMode == 2>(M, sc, sv, P, from, to, e, G, c, ws, st);
            else bad |= process_chunk(M, sc, sv, P, from, to, e, G, c, ws, P.compute_clearance ? &cm : nullptr, st);
            emin = fminf(emin, cm);
            if (bad && !P.compute_clearance) break;
        }
        if (lane == 0) {
            valid[e] = bad ? 0 : 1;
            cost[e] = bad ? FLT_MAX : len;
            if (clearance) clearance[e] = P.compute_clearance ? emin : FLT_MAX;
        }
    }
    flush_stats(stats, st);
}

// ---------------------------------------------------------------------------
// Persistent path
// ---------------------------------------------------------------------------
// n_dev (optional): device-resident edge count overriding n_edges, so a
// captured graph can be replayed with a different number of edges.
// Per-edge preparation of the persistent path, over the grid-stride edges
// of this thread: sample count G, length, cleared per-edge state, and the
// header's maxima and counts (one atomic per warp). The time budget starts
// here, when the call's first kernel runs. Every thread of the grid calls it.
// With lst, the edges that have more than one chunk round are also appended
// to lst (in any order; hdr->n_long counts them), so that the queue's rounds
// >= 1 visit only those edges instead of every edge.
__device__ __forceinline__ void prep_edges(const ps_edge_params& P, const float* __restrict__ from,
                                           const float* __restrict__ to, const int* __restrict__ given,
                                           int n_edges, int D, EdgeWs* hdr, int* G_out, float* len_out, int* bad,
                                           int* clr, int* done, int* lst) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
        hdr->deadline = P.time_budget_ms > 0.0f
                            ? global_ns() + (unsigned long long)((double)P.time_budget_ms * 1.0e6) + 1ull
                            : 0ull;
    int local_max = 0, local_ne = 0;
    unsigned long long local_ns = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_edges; e += gridDim.x * blockDim.x) {
        const float* a = from + (size_t)e * D;
        const float* b = to + (size_t)e * D;
        const float len = edge_length(a, b, D);
        const int G = edge_samples(P, given, e, a, b, D, len);
        G_out[e] = G;
        len_out[e] = len;
        bad[e] = 0;
        clr[e] = ordered_float(FLT_MAX);
        done[e] = 0;
        const int rounds = ChunkOrder(G).rounds();
        local_max = max(local_max, rounds);
        local_ns += (unsigned long long)(G + ((G % 16) != 0 ? 1 : 0));
        local_ne += G > 0;
        if (lst) {   // one atomic per group of converged lanes
            const unsigned am = __activemask();
            const unsigned lb = __ballot_sync(am, rounds > 1);
            const int lane = threadIdx.x & 31, leader = __ffs(am) - 1;
            int base = 0;
            if (lane == leader && lb) base = atomicAdd(&hdr->n_long, __popc(lb));
            base = __shfl_sync(am, base, leader);
            if (rounds > 1) lst[base + __popc(lb & ((1u << lane) - 1u))] = e;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        local_max = max(local_max, __shfl_xor_sync(kFull, local_max, o));
        local_ns += __shfl_xor_sync(kFull, local_ns, o);
        local_ne += __shfl_xor_sync(kFull, local_ne, o);
    }
    if ((threadIdx.x & 31) == 0 && local_max > 0) atomicMax(&hdr->max_rounds, local_max);
    if ((threadIdx.x & 31) == 0 && P.check_self && local_ns > 0) {
        atomicAdd(&hdr->self_samples, local_ns);
        atomicAdd(&hdr->self_edges, local_ne);
    }
}

__global__ void edges_prep_kernel(ps_edge_params P, const float* __restrict__ from, const float* __restrict__ to,
                                  const int* __restrict__ given, int n_edges, int D, EdgeWs* hdr, int* G_out,
                                  float* len_out, int* bad, int* clr, int* done, const int* n_dev = nullptr,
                                  int* lst = nullptr) {
    if (n_dev) n_edges = *n_dev;
    prep_edges(P, from, to, given, n_edges, D, hdr, G_out, len_out, bad, clr, done, lst);
}

// ---------------------------------------------------------------------------
// End-sample probe (persistent path, boxes-only fast variant)
// ---------------------------------------------------------------------------
// Before the chunk queue starts, one thread per edge checks the edge's last
// sample (j = G, t = 1, formed as the chunk path forms it) and retires the
// edge on a hit (bad[e] = 1). The verdict is the OR over the samples, so
// checking one of them first changes no result; the queue skips retired
// edges. A warp chunk costs 32 lanes for an edge that collides at its end
// sample, the probe one lane: on uniformly drawn edges about 85 % of the
// colliding ones collide there. The probe is best effort: a lane whose joint
// reaches more than kProbeCand boxes stops and leaves its edge to the queue.
constexpr int kProbeThreads = 128;
constexpr int kProbeCand = 32;                 // candidate boxes a lane keeps for one joint
constexpr int kProbeStride = kProbeCand + 2;   // 17 words per lane: lanes hit distinct banks

// The fast chunk verdict (process_chunk_fast) for one configuration held by
// one thread: per joint, the boxes within reach of the joint's bound sphere
// (same guarded limits, radius of one sample), the exact spheres 4 per box
// load against them, the approximate gate only after an exact hit. Returns
// true on a confirmed hit, false when none was found or the lane gave up.
template <bool kStats>
__device__ bool lane_probe_hit(const ModelSmem& M, const SceneSmem& sc, const float4* __restrict__ obs,
                               uint16_t* cand, const float* qc, float margin, LaneStats& st) {
    const int NJ = M.H->n_joints;
    Affine T;
    affine_identity(T);
    for (int p = 0; p < NJ; ++p) {
        const JointRec& jr = M.J[p];
        if (p > 0) {
            const float qi = jr.dof >= 0 ? qc[jr.dof] : 0.0f;
            if (jr.parent_slot == 0) {
                Affine I;
                affine_identity(I);
                joint_compose<true>(jr, qi, I, T);
            } else {
                joint_compose<true>(jr, qi, T, T);   // rows are read before they are written
            }
            if (kStats) st.v[ST_JOINTS] += 1;
        }
        if (jr.bound.w < 0.0f) continue;
        float cx, cy, cz;
        sphere_world(T, jr.bound.x, jr.bound.y, jr.bound.z, cx, cy, cz);
        const float Sm = fmaxf(fabsf(cx), fmaxf(fabsf(cy), fabsf(cz)));
        float Rc = jr.bound.w + fmaxf(margin, 0.0f);
        Rc += 4.0f * (Sm + Rc + sc.Bmax + 1.0f) * PS_GUARD_K;
        const float Rcl = Rc * sc.Mscale;   // world radius -> box-frame radius (map stretch)
        const float Rc2 = Rcl * Rcl;
        const float Rj = (Rc * (1.0f + 4.0f * PS_GUARD_K) + 4.0f * PS_GUARD_K * (Sm + 1.0f)) * (1.0f + 1.0e-6f);
        int ncand = 0;
        int o = 0;
        // circumscribed-sphere tests 4 boxes at a time (independent, so they
        // overlap), the box distance for the ones that pass
#pragma unroll 1
        for (; o + 4 <= sc.n_obbs; o += 4) {
            unsigned pass = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float4 ob = obs[o + i];
                const float ex = ob.x - cx, ey = ob.y - cy, ez = ob.z - cz;
                const float lim = Rj + ob.w;   // see box_limits
                pass |= (fmaf(ez, ez, fmaf(ey, ey, ex * ex)) < lim * lim ? 1u : 0u) << i;
            }
            if (kStats) st.v[ST_CULL] += 4;
            while (pass) {
                const int oo = o + __ffs(pass) - 1;
                pass &= pass - 1;
                float qx, qy, qz;
                if (fast_box_dsq(sc.obbs[oo], cx, cy, cz, qx, qy, qz) >= Rc2) continue;
                if (ncand == kProbeCand) return false;   // too many: the queue takes this edge
                cand[ncand++] = (uint16_t)oo;
            }
        }
#pragma unroll 1
        for (; o < sc.n_obbs; ++o) {
            const float4 ob = obs[o];
            const float ex = ob.x - cx, ey = ob.y - cy, ez = ob.z - cz;
            const float lim = Rj + ob.w;
            if (kStats) st.v[ST_CULL] += 1;
            if (fmaf(ez, ez, fmaf(ey, ey, ex * ex)) >= lim * lim) continue;
            float qx, qy, qz;
            if (fast_box_dsq(sc.obbs[o], cx, cy, cz, qx, qy, qz) >= Rc2) continue;
            if (ncand == kProbeCand) return false;
            cand[ncand++] = (uint16_t)o;
        }
        if (ncand == 0) continue;
        const float g = (Sm + jr.bound.w + sc.Bmax + 1.0f) * PS_GUARD_K;
        bool ex = false;
        int k = jr.sph_beg;
        for (; k + 4 <= jr.sph_end && !ex; k += 4) {
            float px[4], py[4], pz[4], sr[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float4 sp = M.S[k + i];
                sphere_world(T, sp.x, sp.y, sp.z, px[i], py[i], pz[i]);
                sr[i] = __fadd_rn(sp.w, margin);
            }
            if (kStats) st.v[ST_SPHERES] += 4;
            ex = spheres_hit<4, kStats>(sc, cand, ncand, px, py, pz, sr, g, st);
        }
        for (; k < jr.sph_end && !ex; ++k) {
            const float4 sp = M.S[k];
            float px, py, pz;
            sphere_world(T, sp.x, sp.y, sp.z, px, py, pz);
            const float sr = __fadd_rn(sp.w, margin);
            if (kStats) st.v[ST_SPHERES] += 1;
            ex = spheres_hit<1, kStats>(sc, cand, ncand, &px, &py, &pz, &sr, g, st);
        }
        if (!ex) continue;
        bool flagged = false;
        for (int a = jr.apx_beg; a < jr.apx_end && !flagged; ++a) {
            const float4 sa = M.A[a];
            float px, py, pz;
            sphere_world(T, sa.x, sa.y, sa.z, px, py, pz);
            const float sr = __fadd_rn(sa.w, margin);
            if (kStats) st.v[ST_SPHERES] += 1;
            flagged = spheres_hit<1, kStats>(sc, cand, ncand, &px, &py, &pz, &sr, g, st);
        }
        if (flagged) return true;
    }
    return false;
}

// Shared memory: model core, staged scene, one configuration per thread, box
// spheres, per-thread candidate lists.
size_t probe_smem_bytes(const ps_model* m, const ps_scene_view* sv) {
    return (size_t)m->dev.bytes_core + scene_smem_bytes(sv) + (size_t)kProbeThreads * m->info.n_dof * 4 +
           (size_t)16 * std::max(sv->n_obbs, 1) + (size_t)kProbeThreads * kProbeStride * 2;
}

// With PrepArgs the kernel also does edges_prep_kernel's work first, over the
// same grid-stride edges (a thread then probes the edges it prepared), which
// saves a launch and overlaps the preparation with the model staging.
struct PrepArgs {
    const int* given;
    float* len;
    int* clr;
    int* done;
    int* lst;   // the long list, or nullptr
};

template <bool kStats, bool kPrep>
__global__ void __launch_bounds__(kProbeThreads, 4) edges_probe_kernel(ModelDev md, ps_scene_view sv,
                                                                        ps_edge_params P,
                                                                        const float* __restrict__ from,
                                                                        const float* __restrict__ to, int n_edges,
                                                                        EdgeWs* hdr, int* Gs,
                                                                        int* bad, unsigned long long* stats,
                                                                        const int* n_dev, PrepArgs pa) {
    if (n_dev) n_edges = *n_dev;
    if (n_edges <= 0) return;
    if (kPrep) {
        const int D = reinterpret_cast<const BlobHeader*>(md.blob)->n_dof;
        prep_edges(P, from, to, pa.given, n_edges, D, hdr, Gs, pa.len, bad, pa.clr, pa.done, pa.lst);
    }
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    if (!stage_model(md, smem, &mbar)) return;   // best effort: the queue still checks every edge
    ObbPrep* obbs = reinterpret_cast<ObbPrep*>(smem + md.bytes_core);
    const int nob = max(sv.n_obbs, 1);
    int* orig = reinterpret_cast<int*>(obbs + nob);
    LayerPrep* layers = reinterpret_cast<LayerPrep*>(orig + ((nob + 3) & ~3));
    SceneSmem sc;
    stage_scene(sv, obbs, orig, layers, counters, &bmax, sc);
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof;
    float* qtile = reinterpret_cast<float*>(layers + PS_MAX_LAYERS);
    float4* obs = reinterpret_cast<float4*>(qtile + kProbeThreads * D);
    uint16_t* cand = reinterpret_cast<uint16_t*>(obs + nob) + threadIdx.x * kProbeStride;
    box_spheres(sc, obs);
    __syncthreads();
    box_limits(sc, obs);
    __syncthreads();
    float* qc = qtile + threadIdx.x * D;
    const unsigned long long deadline = *((volatile unsigned long long*)&hdr->deadline);
    LaneStats st;
    st.zero();
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_edges; e += gridDim.x * blockDim.x) {
        const int G = Gs[e];
        if (G <= 0) continue;
        if (deadline && global_ns() > deadline) break;   // the queue reports the timeout
        const float t = __fdiv_rn((float)G, (float)G);   // sample j = G, as process_chunk forms it
        const float* a = from + (size_t)e * D;
        const float* b = to + (size_t)e * D;
        for (int i = 0; i < D; ++i) {
            const float ai = __ldg(a + i), bi = __ldg(b + i);
            qc[i] = __fmaf_rn(t, __fadd_rn(bi, -ai), ai);
        }
        if (kStats) st.v[ST_SAMPLES] += 1;
        if (lane_probe_hit<kStats>(M, sc, obs, cand, qc, P.collision_margin, st)) bad[e] = 1;
    }
    flush_stats(stats, st);
}

// Kernel, shared memory and grid of the probe for edge variant `mode`, or
// none: the probe serves the boxes-only fast variant (the generic one serves
// clearance, which wants every sample, and masks; the ESDF lookups do not pay
// off one lane at a time) with enough edges to fill the GPU. `share` scales
// the grid (mixed batch).
struct ProbePlan {
    // k: the probe alone (the preparation ran before it); kp: preparation and
    // probe in one launch. Same shared memory and grid.
    void (*k)(ModelDev, ps_scene_view, ps_edge_params, const float*, const float*, int, EdgeWs*, int*, int*,
              unsigned long long*, const int*, PrepArgs) = nullptr;
    void (*kp)(ModelDev, ps_scene_view, ps_edge_params, const float*, const float*, int, EdgeWs*, int*, int*,
               unsigned long long*, const int*, PrepArgs) = nullptr;
    size_t smem = 0;
    int grid = 1;
};

int plan_probe(const ps_model* m, const ps_scene_view* sv, int mode, bool stats, float share, int max_edges,
               int choice, ProbePlan& out) {
    out = ProbePlan{};
    if (mode != 1 || max_edges <= 0 || sv->n_obbs == 0 || choice == 2) return PS_OK;
    // One thread per edge: below 8 warps per SM the probe runs latency-bound
    // and costs more than it retires (measured: the 16 K segment edges of a
    // 256-request CHOMP iteration ran 3 % slower with it). choice 1 forces it.
    if (choice != 1 && (long long)max_edges < 8ll * 32 * sm_count()) return PS_OK;
    out.k = stats ? edges_probe_kernel<true, false> : edges_probe_kernel<false, false>;
    out.kp = stats ? edges_probe_kernel<true, true> : edges_probe_kernel<false, true>;
    out.smem = probe_smem_bytes(m, sv);
    PS_TRY_CUDA(allow_smem((const void*)out.k, out.smem));
    PS_TRY_CUDA(allow_smem((const void*)out.kp, out.smem));
    int per_sm = 0;
    PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, out.k, kProbeThreads, out.smem));
    if (per_sm < 1) return set_error(PS_EINVAL, "edge probe kernel does not fit on an SM with this scene");
    const int cap = (max_edges + kProbeThreads - 1) / kProbeThreads;
    out.grid = std::max(1, std::min(cap, (int)(share * sm_count() * per_sm + 0.5f)));
    return PS_OK;
}

// Residency per variant, measured: the boxes-only fast path runs fastest
// with 5 blocks per SM (room for 96 registers), the ESDF variant with 6.
template <int kMode, bool kStats>
__global__ void __launch_bounds__(kEdgeThreads, kMode == 1 ? 5 : (kMode ? 6 : 3)) edges_queue_kernel(ModelDev md, ps_scene_view sv, ps_edge_params P,
                                                                  const float* __restrict__ from,
                                                                  const float* __restrict__ to, int n_edges,
                                                                  EdgeWs* hdr, const int* __restrict__ Gs, int* bad,
                                                                  int* clr, int* done, unsigned long long* stats,
                                                                  int pass, const int* n_dev = nullptr,
                                                                  const int* __restrict__ lst = nullptr) {
    if (n_dev) n_edges = *n_dev;
    // Rounds of this launch. With many edges per resident warp (>= 8) one
    // launch (pass 0) runs every round and pass 1 returns at once. With fewer,
    // round 1 would start while much of round 0 is still in flight and check
    // chunks of edges that round 0 retires, so pass 0 runs round 0 only and
    // the second launch (pass 1) the rest.
    const int max_rounds = *((volatile int*)&hdr->max_rounds);
    const bool split = (long long)n_edges < 8ll * gridDim.x * kWarps;
    const int r_lo = pass == 0 ? 0 : (split ? 1 : max_rounds);
    const int r_hi = pass == 0 ? (split ? min(max_rounds, 1) : max_rounds) : max_rounds;
    // Chunk-major item space. With the long list (lst): round 0 of every edge
    // (when this pass runs round 0), then rounds k_lo .. r_hi - 1 of the listed
    // edges only, since an edge with one round has nothing after round 0.
    // Without it: rounds r_lo .. r_hi - 1 of every edge.
    const long long n_long = lst ? (long long)*((volatile int*)&hdr->n_long) : (long long)n_edges;
    const long long items0 = (lst && r_lo == 0 && r_hi >= 1) ? (long long)n_edges : 0ll;
    const int k_lo = lst ? max(r_lo, 1) : r_lo;
    const long long itemsL = r_hi > k_lo ? (long long)(r_hi - k_lo) * n_long : 0ll;
    const long long total = items0 + itemsL;
    if (total == 0) return;   // uniform over the grid: nothing staged yet
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    if (!stage_model(md, smem, &mbar)) {
        // fail closed: finalize reports every edge that is neither retired
        // nor complete as invalid, and the status query PS_ETIMEOUT
        if (threadIdx.x == 0) atomicExch(&hdr->timed_out, 1);
        return;
    }
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof;
    EdgeSmem es = carve(smem, md, sv, D);
    SceneSmem sc;
    stage_scene(sv, es.obbs, es.orig, es.layers, counters, &bmax, sc);
    box_spheres(sc, es.obs);
    __syncthreads();
    box_limits(sc, es.obs);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nob_pad = (max(sv.n_obbs, 1) + 7) & ~7;
    WarpScratch ws{es.q + warp * 32 * D, es.cand + warp * nob_pad, es.obs};
    LaneStats st;
    st.zero();
    unsigned long long* head = &hdr->head[pass == 0 ? 0 : 1];
    // time budget: stop pulling items past the deadline (checked per grab)
    const unsigned long long deadline = *((volatile unsigned long long*)&hdr->deadline);
    // Items per grab: up to 32, fewer when the pass has few items, so that
    // every resident warp gets a share.
    const int grab = P.grab > 0 ? min(P.grab, 32)
                                : (int)max(1ll, min(32ll, total / ((long long)gridDim.x * kWarps * 2)));
    volatile int* vbad = bad;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) {
            if (deadline && global_ns() > deadline) {
                atomicExch(&hdr->timed_out, 1);
                base = (unsigned long long)total;   // stop this warp
            } else {
                base = atomicAdd(head, (unsigned long long)grab);
            }
        }
        base = __shfl_sync(kFull, base, 0);
        if ((long long)base >= total) break;
        // Each lane inspects one item; live items are processed by the whole warp.
        const long long item = (long long)base + lane;
        int e = -1, k = 0, G = 0;
        bool live = false;
        if (lane < grab && item < total) {
            if (item < items0) {
                k = 0;
                e = (int)item;
            } else {
                const long long i2 = item - items0;
                int idx;
                if (i2 < (1ll << 31)) {   // 32-bit division in the common case
                    k = (int)((unsigned)i2 / (unsigned)n_long);
                    idx = (int)((unsigned)i2 - (unsigned)k * (unsigned)n_long);
                } else {
                    k = (int)(i2 / n_long);
                    idx = (int)(i2 - (long long)k * n_long);
                }
                k += k_lo;
                e = lst ? __ldg(lst + idx) : idx;
            }
            G = __ldg(Gs + e);
            const ChunkOrder ord(G);
            if (k < ord.rounds()) {
                k = ord.chunk(k);   // round -> chunk index
                // a retired edge's remaining chunks still count toward the
                // clearance, which covers every sample (edge_eval.cuh:133-153)
                live = k < ord.nc && (P.compute_clearance || vbad[e] == 0);
            }
        }
        unsigned todo = __ballot_sync(kFull, live);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const int ee = __shfl_sync(kFull, e, src);
            const int kk = __shfl_sync(kFull, k, src);
            const int GG = __shfl_sync(kFull, G, src);
            int retired = 0;
            if (lane == 0) retired = vbad[ee];
            retired = __shfl_sync(kFull, retired, 0);
            if (!P.compute_clearance && retired) continue;   // retired meanwhile
            float cm = FLT_MAX;
            const bool h = kMode ? process_chunk_fast<kStats, kMode == 2>(M, sc, sv, P, from, to, ee, GG, kk, ws, st)
                                 : process_chunk(M, sc, sv, P, from, to, ee, GG, kk, ws,
                                                 P.compute_clearance ? &cm : nullptr, st);
            if (lane == 0) {
                if (h) vbad[ee] = 1;
                if (P.compute_clearance) atomicMin(clr + ee, ordered_float(cm));
                if (deadline) atomicAdd(done + ee, 1);   // completed chunks, read only after a timeout
            }
        }
    }
    flush_stats(stats, st);
}

// Self-collision pass of the edge checks (check_self: edge_eval.cuh:128 runs
// two_phase_cc with params.check_self for every sample). After the scene
// pass, each edge without a scene hit gets the self verdict (lane_self_hit)
// of every sample of the scene pass' set: t = j/G for j = 1..G, and j = 0
// when G % 16 != 0. A block takes a window of W consecutive edges, lays
// their samples end to end and checks them kSelfThreads at a time, one per
// thread; an edge's remaining samples are skipped after its first hit. W is
// sized from the counts the prep kernel took (about kSelfThreads samples per
// window over the edges that have samples): short edges share a block
// instead of leaving its threads idle, long edges get a block each so that
// every SM has work. With a workspace, blocks take windows from a counter.
// Persistent mode (bad != nullptr): bad[e] goes from 0 to 1 (self hit) or 2
// (checked, free); an edge still at 0 after a deadline comes back invalid.
// Plain mode (valid, cost): a self hit turns a free edge invalid.
__global__ void __launch_bounds__(kSelfThreads, 6) edges_self_kernel(ModelDev md, ps_edge_params P,
                                                                  const float* __restrict__ from,
                                                                  const float* __restrict__ to,
                                                                  const int* __restrict__ given, int n_edges,
                                                                  const int* __restrict__ Gs, int* bad,
                                                                  uint8_t* valid, float* cost, EdgeWs* hdr,
                                                                  unsigned long long* stats,
                                                                  const int* n_dev = nullptr) {
    static_assert(kSelfThreads == 64, "two-warp scan below");
    if (n_dev) n_edges = *n_dev;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int s_off[kSelfThreads + 1], s_G[kSelfThreads], s_hit[kSelfThreads], s_wsum[2], s_stop;
    if (!stage_model(md, smem, &mbar)) {
        // fail closed. Persistent: bad[] stays 0 for the edges no block
        // checked, and finalize reports them invalid once timed_out is set.
        // Plain: this block's windows (8 edges each) come back invalid.
        if (hdr) {
            if (threadIdx.x == 0) atomicExch(&hdr->timed_out, 1);
        } else if (!bad) {
            for (long long e0 = (long long)blockIdx.x * 8; e0 < n_edges; e0 += (long long)gridDim.x * 8)
                if (threadIdx.x < 8 && e0 + threadIdx.x < n_edges) {
                    valid[e0 + threadIdx.x] = 0;
                    cost[e0 + threadIdx.x] = FLT_MAX;
                }
        }
        return;
    }
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof, NA = M.H->n_approx, NJ = M.H->n_joints;
    const SelfFrames sm = carve_self_frames<kSelfThreads>(smem + md.bytes_core, NA, NJ, md.bound_from_apx != 0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float* qc = sm.end + tid * D;
    const bool persistent = bad != nullptr;
    const unsigned long long deadline = hdr ? *((volatile unsigned long long*)&hdr->deadline) : 0ull;
    LaneStats st;
    st.zero();
    bool stopped = false;
    int W = 8;   // plain path: no sample count
    if (hdr) {
        const unsigned long long tot = *((volatile unsigned long long*)&hdr->self_samples);
        const unsigned long long ne = (unsigned long long)*((volatile int*)&hdr->self_edges);
        W = tot > 0 ? (int)min(64ull, max(1ull, (64ull * ne + tot - 1) / tot)) : 64;
    }
    __shared__ int s_win;
    for (int wi = blockIdx.x;; wi += gridDim.x) {
        if (hdr) {   // dynamic: the next window from the counter
            __syncthreads();
            if (tid == 0) s_win = atomicAdd(&hdr->self_next, 1);
            __syncthreads();
            wi = s_win;
        }
        const long long w0l = (long long)wi * W;
        if (w0l >= n_edges || stopped) break;
        const int w0 = (int)w0l;
        const int e = w0 + tid;
        const bool active = tid < W && e < n_edges && (persistent ? bad[e] == 0 : valid[e] != 0);
        int G = 0;
        if (active) {
            const float* a = from + (size_t)e * D;
            const float* b = to + (size_t)e * D;
            G = persistent ? Gs[e] : edge_samples(P, given, e, a, b, D, edge_length(a, b, D));
        }
        const int ns = active ? G + ((G % 16) != 0 ? 1 : 0) : 0;
        int v = ns;   // inclusive scan over the block's 64 edges
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, v, o);
            if (lane >= o) v += y;
        }
        if (lane == 31) s_wsum[warp] = v;
        s_G[tid] = G;
        s_hit[tid] = 0;
        __syncthreads();
        s_off[tid + 1] = v + (warp == 1 ? s_wsum[0] : 0);
        if (tid == 0) s_off[0] = 0;
        __syncthreads();
        const int total = s_off[kSelfThreads];
        for (int base = 0; base < total; base += kSelfThreads) {
            if (deadline) {
                if (tid == 0) s_stop = global_ns() > deadline;
                __syncthreads();
                if (s_stop) {
                    if (tid == 0) atomicExch(&hdr->timed_out, 1);
                    stopped = true;
                    break;
                }
            }
            const int idx = base + tid;
            if (idx < total) {
                int lo = 0, hi = kSelfThreads;   // s_off[lo] <= idx < s_off[hi]
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_off[mid] <= idx) lo = mid;
                    else hi = mid;
                }
                if (!*((volatile int*)&s_hit[lo])) {
                    const int k = idx - s_off[lo], Gl = s_G[lo], el = w0 + lo;
                    const int j = k < Gl ? k + 1 : 0;
                    const float t = __fdiv_rn((float)j, (float)Gl);
                    const float* a = from + (size_t)el * D;
                    const float* b = to + (size_t)el * D;
                    for (int i = 0; i < D; ++i) {
                        const float ai = __ldg(a + i), bi = __ldg(b + i);
                        qc[i] = __fmaf_rn(t, __fadd_rn(bi, -ai), ai);
                    }
                    st.v[ST_SAMPLES] += 1;
                    if (lane_self_hit<kSelfThreads>(M, md, qc, sm, tid, st)) s_hit[lo] = 1;
                }
            }
            __syncthreads();
        }
        if (active && !stopped) {
            if (persistent) {
                bad[e] = s_hit[tid] ? 1 : 2;
            } else if (s_hit[tid]) {
                valid[e] = 0;
                cost[e] = FLT_MAX;
            }
        }
        __syncthreads();   // the next window rewrites the block's tables
    }
    flush_stats(stats, st);
}

// After a timeout an edge that is neither retired nor complete comes back
// invalid (cost FLT_MAX): not shown free. Its clearance is the min over the
// samples that were checked. With check_self an edge is free only when the
// self pass marked it so (bad == 2).
__global__ void edges_finalize_kernel(int n_edges, const ps_edge_params P, const int* __restrict__ bad,
                                      const float* __restrict__ len, const int* __restrict__ clr,
                                      const int* __restrict__ done, const int* __restrict__ Gs, const EdgeWs* hdr,
                                      uint8_t* __restrict__ valid, float* __restrict__ cost,
                                      float* __restrict__ clearance, const int* n_dev = nullptr) {
    if (n_dev) n_edges = *n_dev;
    const bool timed_out = hdr->timed_out != 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_edges; e += gridDim.x * blockDim.x) {
        const int bv = bad[e];
        const bool b = (P.check_self ? bv != 2 : bv != 0) || (timed_out && done[e] < ChunkOrder(Gs[e]).nc);
        valid[e] = b ? 0 : 1;
        cost[e] = b ? FLT_MAX : len[e];
        if (clearance) clearance[e] = P.compute_clearance ? unordered_float(clr[e]) : FLT_MAX;
    }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Launches the self pass when params ask for it (a no-op otherwise). The grid
// covers every SM at the kernel's occupancy; blocks stride over the edges.
int launch_edges_self(const ps_model* m, const ps_edge_params* P, const float* from, const float* to,
                      const int* given, int n_edges, const int* Gs, int* bad, uint8_t* valid, float* cost,
                      EdgeWs* hdr, const int* n_dev, cudaStream_t s) {
    if (!P->check_self || n_edges <= 0) return PS_OK;
    if (int rc = check_self_fits(m)) return rc;
    const size_t smem = self_lane_smem_bytes(m);
    PS_TRY_CUDA(allow_smem((const void*)edges_self_kernel, smem));
    int per_sm = 0;
    PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, edges_self_kernel, kSelfThreads, smem));
    if (per_sm < 1) return set_error(PS_EINVAL, "self-check kernel does not fit on an SM with this model");
    const int grid = std::max(1, std::min(n_edges, sm_count() * per_sm));
    edges_self_kernel<<<grid, kSelfThreads, smem, s>>>(m->dev, *P, from, to, given, n_edges, Gs, bad, valid, cost,
                                                       hdr, g_stats, n_dev);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}



// Kernel variant: 0 generic, 1 fast (boxes only), 2 fast with ESDF layers.
// The self check (check_self) is a separate pass (edges_self_kernel) after
// either variant.
int fast_path(const ps_model* m, const ps_scene_view* sv, const ps_edge_params* P) {
    // (sphere_obb_acm_mask_approx changes no result: the approximate gate applies no mask)
    const bool fast = m->info.approx_shares_chain && m->root_slot_only && !P->compute_clearance &&
                      !sv->sphere_obb_acm_mask && !sv->sphere_acm_mask;
    return fast ? (sv->n_voxel_layers > 0 ? 2 : 1) : 0;
}

template <typename K>
K pick(int mode, bool stats, K g0, K g1, K f0, K f1, K e0, K e1) {
    if (mode == 2) return stats ? e1 : e0;
    if (mode == 1) return stats ? f1 : f0;
    return stats ? g1 : g0;
}

}  // namespace
}  // namespace ps
