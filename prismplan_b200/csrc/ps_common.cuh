// ps_common.cuh -- device-side building blocks of the sm_100a substrate.
//
// Arithmetic that decides a collision Boolean reproduces the reference's FP32
// operation sequence exactly (paths inside code/gpu_planning/cpp/src/):
//   * joint step columns      planning/utils.cuh:571-699 (xrot_fn/yrot_fn/zrot_fn/prism_fn)
//   * 4x4 compose             planning/runtime_kinematics.cuh:60-70 with dot4_col (utils.cuh:709-711)
//   * sphere emission         planning/runtime_kinematics.cuh:74-85
//   * world -> box frame      collision/scene_collision.cuh:24-51
//   * sphere-vs-box Boolean   collision/scene_collision.cuh:59-78
//   * ESDF nearest lookup     collision/scene_collision.cuh:192-331
// nvcc contracts `a*b + c*d` into fma(a, b, c*d) (the left product is fused,
// the right one rounded). The FP32 expressions below spell that sequence out
// with __fmaf_rn / __fmul_rn / __fadd_rn (through fma_ab_cd for every
// two-product sum) so it no longer depends on how the compiler contracts this
// file; the GPU parity tests compare the results bitwise against the
// reference kernels.
//
// Everything here is FP32 CUDA-core arithmetic: the 4x4 chains and the
// per-pair distances are not dense contractions, so tensor cores do not apply.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/prism_b200.h"

namespace ps {

// ---------------------------------------------------------------------------
// Model blob layout (device, one allocation, built by ps_model_create)
// ---------------------------------------------------------------------------
struct BlobHeader {          // 64 bytes
    int n_dof, n_joints, n_spheres, n_approx;
    int n_self_pairs, n_apx_self_pairs, approx_shares_chain, n_t_slots;
    int off_joints, off_apx_joints, off_spheres, off_sph_orig;
    int off_apx, off_apx_orig, bytes_core, bytes_total;
};

// One joint in DFS visit order (112 bytes).
struct JointRec {
    float ft[12];            // rows 0..2 of the fixed transform, row-major
    int type, dof, parent_slot, slot;
    int sph_beg, sph_end, apx_beg, apx_end;   // ranges into the reordered tables
    float4 bound;            // link-frame point + radius enclosing every exact and
                             // approximate sphere of the joint (w < 0: none)
    int parent_pos;          // DFS position of the parent joint (root: 0)
    int pad[3];
};

// Self pairs (global memory): packed (i | j << 16), reordered sphere indices.
// The same pairs as runs: sruns[r] = (i | q << 9 | len << 14, j0) is sphere i
// against the len consecutive spheres j0..j0+len-1 of joint q (DFS position).
// Runs are ordered by joint pair (joint of i, q), then i, then j0;
// sjp[k] = (a | q << 16, first run, end run, 0) lists the joint pairs, nearest
// in DFS order (|q - a|) first.
// Limits (global memory): lower[n_dof], upper[n_dof].
struct ModelDev {
    const unsigned char* blob;     // device
    const uint32_t* self_pairs;    // device
    const uint32_t* apx_self_pairs;// device
    const uint2* sruns;            // device, self-pair runs
    int n_sruns;
    const uint4* sjp;              // device, joint pairs: (a | q << 16, first run, end run, 0)
    int n_sjp;
    int bound_from_apx;            // 1: every joint with exact spheres has an approximate sphere on the same
                                   // chain, whose centre is the joint's bound centre (the self check reads it there)
    const float* lower;            // device
    const float* upper;            // device
    int* status;                   // device error latch
    int bytes_core;
    int stage_polls;               // polls of the staging wait before a kernel gives up
};

// Default staging wait: ~2^22 polls, each try_wait may suspend for a
// hardware-defined interval (far beyond any real copy of a few KB).
#define PS_STAGE_POLLS (1 << 22)

// ---------------------------------------------------------------------------
// Prepared obstacle tables in shared memory
// ---------------------------------------------------------------------------
// Box o: l = R p + t is the world->box map of the reference's quaternion
// formula (v + qw t + q x t, t = 2 q x v, which is linear in v), so R is that
// map's matrix for the stored (possibly slightly non-unit) quaternion.
struct ObbPrep {             // 80 bytes
    float4 r0, r1, r2;       // rows of R, .w = translation (pose[0..2])
    float4 h;                // half extents (dims * 0.5, exact), .w = |t|inf + |h|inf
    float4 q;                // stored quaternion (qw, qx, qy, qz) for the exact path
};

struct LayerPrep {           // one ESDF layer, 64 bytes
    float4 params;           // dx, dy, dz, voxel_size
    float4 t;                // translation, .w = inv_vs
    float4 q;                // qw, qx, qy, qz
    int nx, ny, nz, enabled;
};

// Guard band of the fast sphere-vs-box path, in metres per metre of
// coordinate magnitude: the fast map (3x3 matrix, 3 FMA per coordinate) and
// the reference quaternion sequence differ by < 1.5e-5 m at the scales used
// (|p|, |t| <= a few metres); the band is (S + B + 1) * PS_GUARD_K with
// PS_GUARD_K = 2^-15 ~ 3.05e-5, leaving a 2x margin over a worst-case
// rounding bound and >10x over typical errors. Pairs whose fast squared
// distance lands inside the band are re-decided with the exact sequence.
#define PS_GUARD_K 3.0517578125e-05f

// ---------------------------------------------------------------------------
// Exact reference arithmetic
// ---------------------------------------------------------------------------
// a*b + c*d as nvcc contracts it: the left product is fused, the right one
// rounded. PS_FUSE_LEFT=0 builds the other order (diagnostic builds only).
#ifndef PS_FUSE_LEFT
#define PS_FUSE_LEFT 1
#endif
__device__ __forceinline__ float fma_ab_cd(float a, float b, float c, float d) {
#if PS_FUSE_LEFT
    return __fmaf_rn(a, b, __fmul_rn(c, d));
#else
    return __fmaf_rn(c, d, __fmul_rn(a, b));
#endif
}

// The 4x4 compose (dot4_col, utils.cuh:709-711): first two products, per
// row r of the result. PS_COMPOSE_RIGHT_ROWS is a bitmask of rows whose right
// product is fused (diagnostic builds only).
#ifndef PS_COMPOSE_RIGHT_ROWS
#define PS_COMPOSE_RIGHT_ROWS 0
#endif
template <int kRow>
__device__ __forceinline__ float compose_sum(float a, float b, float c, float d) {
    if ((PS_COMPOSE_RIGHT_ROWS >> kRow) & 1) return __fmaf_rn(c, d, __fmul_rn(a, b));
    return __fmaf_rn(a, b, __fmul_rn(c, d));
}

// The joint-step columns (utils.cuh:571-699, `ft[x] * f1 + f2 * ft[y]` per
// row r of the step) come out of nvcc with a row-dependent contraction,
// measured on B200 against the reference kernels for every joint type and
// column: row 0 fuses the right product, fma(f2, ft[y], rn(ft[x]*f1)); rows 1
// and 2 fuse the left one, fma(ft[x], f1, rn(f2*ft[y])).
template <int kRow>
__device__ __forceinline__ float step_sum(float a, float b, float c, float d) {
    if (kRow == 0) return __fmaf_rn(c, d, __fmul_rn(a, b));
    return __fmaf_rn(a, b, __fmul_rn(c, d));
}

// transform_sphere_to_local (scene_collision.cuh:24-51), exact sequence.
__device__ __forceinline__ void ref_to_local(float qw, float qx, float qy, float qz, float t0, float t1,
                                             float t2, float sx, float sy, float sz, float& lx, float& ly,
                                             float& lz) {
    float tx = __fmul_rn(2.0f, fma_ab_cd(qy, sz, -qz, sy));
    float ty = __fmul_rn(2.0f, fma_ab_cd(qz, sx, -qx, sz));
    float tz = __fmul_rn(2.0f, fma_ab_cd(qx, sy, -qy, sx));
    float rx = __fadd_rn(__fmaf_rn(qw, tx, sx), fma_ab_cd(qy, tz, -qz, ty));
    float ry = __fadd_rn(__fmaf_rn(qw, ty, sy), fma_ab_cd(qz, tx, -qx, tz));
    float rz = __fadd_rn(__fmaf_rn(qw, tz, sz), fma_ab_cd(qx, ty, -qy, tx));
    lx = __fadd_rn(rx, t0);
    ly = __fadd_rn(ry, t1);
    lz = __fadd_rn(rz, t2);
}

// sphere_single_obb_collision (scene_collision.cuh:59-78), exact sequence;
// also returns the squared outside distance it compared.
__device__ __forceinline__ bool ref_obb_hit(const ObbPrep& o, float sx, float sy, float sz, float sr) {
    float lx, ly, lz;
    ref_to_local(o.q.x, o.q.y, o.q.z, o.q.w, o.r0.w, o.r1.w, o.r2.w, sx, sy, sz, lx, ly, lz);
    float cx = fmaxf(0.0f, __fadd_rn(fabsf(lx), -o.h.x));
    float cy = fmaxf(0.0f, __fadd_rn(fabsf(ly), -o.h.y));
    float cz = fmaxf(0.0f, __fadd_rn(fabsf(lz), -o.h.z));
    float dsq = __fmaf_rn(cz, cz, fma_ab_cd(cx, cx, cy, cy));
    return dsq < __fmul_rn(sr, sr);
}

// Sphere-sphere overlap (utils.cuh:239-267): sum - (ar+br)^2 < 0 with the
// subtraction contracted, i.e. fma(-rs, rs, sum) < 0.
__device__ __forceinline__ bool ref_self_hit(float ax, float ay, float az, float ar, float bx, float by,
                                             float bz, float br) {
    float xs = __fadd_rn(ax, -bx), ys = __fadd_rn(ay, -by), zs = __fadd_rn(az, -bz);
    float sum = __fmaf_rn(zs, zs, fma_ab_cd(xs, xs, ys, ys));
    float rs = __fadd_rn(ar, br);
    return __fmaf_rn(-rs, rs, sum) < 0.0f;
}

// ---------------------------------------------------------------------------
// Forward kinematics: 3x4 affine per joint, held in registers.
// ---------------------------------------------------------------------------
struct Affine {
    float m[12];   // row-major rows 0..2
};

__device__ __forceinline__ void affine_identity(Affine& T) {
#pragma unroll
    for (int k = 0; k < 12; ++k) T.m[k] = (k % 5 == 0) ? 1.0f : 0.0f;
}

// Rotation columns of step row kRow (utils.cuh:571-659).
template <int kRow>
__device__ __forceinline__ void step_rot_row(const JointRec& J, int type, float cs, float sn, float nsn, float* s) {
    const float f0 = J.ft[kRow * 4 + 0], f1 = J.ft[kRow * 4 + 1], f2 = J.ft[kRow * 4 + 2];
    if (type == PS_Z_ROT) {
        s[kRow * 4 + 0] = step_sum<kRow>(f0, cs, sn, f1);
        s[kRow * 4 + 1] = step_sum<kRow>(f0, nsn, cs, f1);
    } else if (type == PS_X_ROT) {
        s[kRow * 4 + 1] = step_sum<kRow>(f1, cs, sn, f2);
        s[kRow * 4 + 2] = step_sum<kRow>(f1, nsn, cs, f2);
    } else {   // PS_Y_ROT
        s[kRow * 4 + 0] = step_sum<kRow>(f0, cs, nsn, f2);
        s[kRow * 4 + 2] = step_sum<kRow>(f0, sn, cs, f2);
    }
}

// Row kRow of P * step (dot4_col); reads the whole parent row first, so the
// output may alias the parent.
template <int kRow>
__device__ __forceinline__ void compose_row(const Affine& P, const float* s, Affine& O) {
    const float p0 = P.m[kRow * 4 + 0], p1 = P.m[kRow * 4 + 1], p2 = P.m[kRow * 4 + 2], p3 = P.m[kRow * 4 + 3];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v = __fmaf_rn(p2, s[8 + c], compose_sum<kRow>(p0, s[c], p1, s[4 + c]));
        O.m[kRow * 4 + c] = (c == 3) ? __fadd_rn(v, p3) : v;
    }
}

// T_out = T_par * step(FT, type, q) with the reference's per-column formulas
// and contraction (utils.cuh:571-711; runtime_kinematics.cuh:60-70). The
// step's row 3 is (0,0,0,1) (validated at model creation), so the fourth
// dot4 term is an exact +0 for rotation columns and +T_par[r][3] for the
// translation column. sn/cs are the joint angle's sine and cosine (read by
// rotation joints only).
__device__ __forceinline__ void joint_compose_sc(const JointRec& J, float qi, float sn, float cs, const Affine& P,
                                                 Affine& O) {
    float s[12];   // step rows 0..2
#pragma unroll
    for (int k = 0; k < 12; ++k) s[k] = J.ft[k];
    const int type = J.type;
    if (type >= PS_X_ROT) {
        const float nsn = -sn;
        step_rot_row<0>(J, type, cs, sn, nsn, s);
        step_rot_row<1>(J, type, cs, sn, nsn, s);
        step_rot_row<2>(J, type, cs, sn, nsn, s);
    } else if (type >= PS_X_PRISM) {
#pragma unroll
        for (int r = 0; r < 3; ++r) s[r * 4 + 3] = __fmaf_rn(J.ft[r * 4 + type], qi, J.ft[r * 4 + 3]);
    }
    // PS_FIXED: step = FT
    compose_row<0>(P, s, O);
    compose_row<1>(P, s, O);
    compose_row<2>(P, s, O);
}

// The same step with its sine/cosine evaluated here: kFastSinCos selects
// __sinf/__cosf (reference, used by every Boolean) or sincosf (accurate, used
// by the cost/gradient path).
template <bool kFastSinCos>
__device__ __forceinline__ void joint_compose(const JointRec& J, float qi, const Affine& P, Affine& O) {
    float sn = 0.0f, cs = 1.0f;
    if (J.type >= PS_X_ROT) {
        if (kFastSinCos) {
            cs = __cosf(qi);
            sn = __sinf(qi);
        } else {
            sincosf(qi, &sn, &cs);
        }
    }
    joint_compose_sc(J, qi, sn, cs, P, O);
}

// World position of a link-frame point (runtime_kinematics.cuh:79-83).
__device__ __forceinline__ void sphere_world(const Affine& T, float x, float y, float z, float& px, float& py,
                                             float& pz) {
    px = __fadd_rn(__fmaf_rn(T.m[2], z, fma_ab_cd(T.m[0], x, T.m[1], y)), T.m[3]);
    py = __fadd_rn(__fmaf_rn(T.m[6], z, fma_ab_cd(T.m[4], x, T.m[5], y)), T.m[7]);
    pz = __fadd_rn(__fmaf_rn(T.m[10], z, fma_ab_cd(T.m[8], x, T.m[9], y)), T.m[11]);
}

// ---------------------------------------------------------------------------
// Fast sphere-vs-box terms (free contraction; used for decisions only through
// the guard band, and directly for clearance / cost values)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fast_box_dsq(const ObbPrep& o, float px, float py, float pz, float& qx,
                                              float& qy, float& qz) {
    float lx = fmaf(o.r0.z, pz, fmaf(o.r0.y, py, fmaf(o.r0.x, px, o.r0.w)));
    float ly = fmaf(o.r1.z, pz, fmaf(o.r1.y, py, fmaf(o.r1.x, px, o.r1.w)));
    float lz = fmaf(o.r2.z, pz, fmaf(o.r2.y, py, fmaf(o.r2.x, px, o.r2.w)));
    qx = fabsf(lx) - o.h.x;
    qy = fabsf(ly) - o.h.y;
    qz = fabsf(lz) - o.h.z;
    float cx = fmaxf(qx, 0.0f), cy = fmaxf(qy, 0.0f), cz = fmaxf(qz, 0.0f);
    return fmaf(cz, cz, fmaf(cy, cy, cx * cx));
}

// Decision thresholds for one sphere: definite hit if dsq < lo, definite
// miss if dsq >= hi, else re-decide exactly. Bmax: max over boxes of
// |t|inf + |h|inf.
__device__ __forceinline__ void guard_thresholds(float px, float py, float pz, float sr, float Bmax, float& lo,
                                                 float& hi) {
    float S = fmaxf(fabsf(px), fmaxf(fabsf(py), fabsf(pz)));
    float g = (S + Bmax + 1.0f) * PS_GUARD_K;
    float a = fmaxf(sr - g, 0.0f), b = sr + g;
    lo = a * a * (1.0f - 1.0e-6f);
    hi = b * b * (1.0f + 1.0e-6f);
}

// ---------------------------------------------------------------------------
// Shared-memory scene staging
// ---------------------------------------------------------------------------
struct SceneSmem {
    const ObbPrep* obbs;       // compacted enabled boxes
    const int* obb_orig;       // original index (ACM masks)
    const LayerPrep* layers;
    int n_obbs;                // enabled count
    int n_layers;
    float Bmax;
    float Mscale;              // bound on |M v| / |v| over the boxes' and layers' world -> local maps
};

// A stored quaternion q with s = |q|^2 != 1 makes the reference's world ->
// local map M = (1 - s) I + s R(q / |q|) instead of a rotation. M is normal
// with singular values 1 and |(1 - s) + s e^{+-i theta}|, so with e = s - 1:
//   |M v| <= (1 + 2|e|) |v|,  |M^-1 v| <= |v| / sqrt(1 - 4|e|(1 + |e|)).
// The broad phases, which bound world distances, widen by these factors; a
// box whose inverse bound does not hold (|e| >= 0.16) is never culled.
__device__ __forceinline__ float quat_norm_err(float qw, float qx, float qy, float qz) {
    return fabsf(fmaf(qw, qw, fmaf(qx, qx, fmaf(qy, qy, qz * qz))) - 1.0f) + 1.0e-6f;   // + its own rounding
}
__device__ __forceinline__ float map_stretch(float e) { return (1.0f + 2.0f * e) * (1.0f + 1.0e-6f); }

// stage_scene / stage_model live in ps_stage.cuh.

// ---------------------------------------------------------------------------
// ESDF lookup (nearest: exact reference sequence; trilinear: new mode)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int robust_floor_dev(float x) {
    // robust_floor_scalar (scene_collision.cuh:192-200)
    float nearest = roundf(x);
    float diff = __fadd_rn(x, -nearest);
    if (diff >= 1e-4f) return __float2int_rd(x);
    return __float2int_rn(nearest);
}

// Returns true and the layer's distance ("positive = inside") if the sphere
// centre maps to an observed voxel inside the 2-voxel guard.
__device__ __forceinline__ bool esdf_sample(const LayerPrep& L, const float* feat, int max_vox, float px,
                                            float py, float pz, int mode, float& dist) {
    if (!L.enabled) return false;
    float lx, ly, lz;
    ref_to_local(L.q.x, L.q.y, L.q.z, L.q.w, L.t.x, L.t.y, L.t.z, px, py, pz, lx, ly, lz);
    const float inv_vs = L.t.w;
    const int B = 2;
    if (mode == PS_ESDF_NEAREST) {
        int ix = (int)__fmul_rn(__fmaf_rn(L.params.x, 0.5f, lx), inv_vs);
        int iy = (int)__fmul_rn(__fmaf_rn(L.params.y, 0.5f, ly), inv_vs);
        int iz = (int)__fmul_rn(__fmaf_rn(L.params.z, 0.5f, lz), inv_vs);
        if (ix >= L.nx - B || iy >= L.ny - B || iz >= L.nz - B || ix <= B || iy <= B || iz <= B) return false;
        long long li = (long long)ix * L.ny * L.nz + (long long)iy * L.nz + iz;
        if (li >= max_vox) return false;
        float d = __ldg(feat + li);
        if (d <= -999.0f) return false;
        dist = d;
        return true;
    }
    float gx = (lx + L.params.x * 0.5f) * inv_vs;
    float gy = (ly + L.params.y * 0.5f) * inv_vs;
    float gz = (lz + L.params.z * 0.5f) * inv_vs;
    float fx0 = floorf(gx), fy0 = floorf(gy), fz0 = floorf(gz);
    if (!(fx0 > (float)B && fy0 > (float)B && fz0 > (float)B && fx0 + 1.0f < (float)(L.nx - B) &&
          fy0 + 1.0f < (float)(L.ny - B) && fz0 + 1.0f < (float)(L.nz - B)))
        return false;
    int ix = (int)fx0, iy = (int)fy0, iz = (int)fz0;
    long long base = (long long)ix * L.ny * L.nz + (long long)iy * L.nz + iz;
    long long sx = (long long)L.ny * L.nz, sy = L.nz;
    if (base + sx + sy + 1 >= max_vox) return false;
    float v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        v[c] = __ldg(feat + base + ((c & 1) ? sx : 0) + ((c & 2) ? sy : 0) + ((c & 4) ? 1 : 0));
        if (v[c] <= -999.0f) return false;
    }
    float fx = gx - fx0, fy = gy - fy0, fz = gz - fz0;
    float x00 = v[0] + fx * (v[1] - v[0]), x10 = v[2] + fx * (v[3] - v[2]);
    float x01 = v[4] + fx * (v[5] - v[4]), x11 = v[6] + fx * (v[7] - v[6]);
    float y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    dist = y0 + fz * (y1 - y0);
    return true;
}

// Trilinear sample with its world-frame gradient d(dist)/dp (the interpolant
// is linear in each cell, so this is the exact derivative inside a cell).
// Same lookup, guard and sentinel rules as esdf_sample in trilinear mode.
__device__ __forceinline__ bool esdf_sample_trilinear_grad(const LayerPrep& L, const float* feat, int max_vox, float px,
                                                           float py, float pz, float& dist, float& gx, float& gy,
                                                           float& gz) {
    if (!L.enabled) return false;
    float lx, ly, lz;
    ref_to_local(L.q.x, L.q.y, L.q.z, L.q.w, L.t.x, L.t.y, L.t.z, px, py, pz, lx, ly, lz);
    const float inv_vs = L.t.w;
    const int B = 2;
    const float ux = (lx + L.params.x * 0.5f) * inv_vs, uy = (ly + L.params.y * 0.5f) * inv_vs,
                uz = (lz + L.params.z * 0.5f) * inv_vs;
    const float fx0 = floorf(ux), fy0 = floorf(uy), fz0 = floorf(uz);
    if (!(fx0 > (float)B && fy0 > (float)B && fz0 > (float)B && fx0 + 1.0f < (float)(L.nx - B) &&
          fy0 + 1.0f < (float)(L.ny - B) && fz0 + 1.0f < (float)(L.nz - B)))
        return false;
    const long long base = (long long)(int)fx0 * L.ny * L.nz + (long long)(int)fy0 * L.nz + (int)fz0;
    const long long sx = (long long)L.ny * L.nz, sy = L.nz;
    if (base + sx + sy + 1 >= max_vox) return false;
    float v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        v[c] = __ldg(feat + base + ((c & 1) ? sx : 0) + ((c & 2) ? sy : 0) + ((c & 4) ? 1 : 0));
        if (v[c] <= -999.0f) return false;
    }
    const float fx = ux - fx0, fy = uy - fy0, fz = uz - fz0;
    const float x00 = v[0] + fx * (v[1] - v[0]), x10 = v[2] + fx * (v[3] - v[2]);
    const float x01 = v[4] + fx * (v[5] - v[4]), x11 = v[6] + fx * (v[7] - v[6]);
    const float y0 = x00 + fy * (x10 - x00), y1 = x01 + fy * (x11 - x01);
    dist = y0 + fz * (y1 - y0);
    // d/d(fx, fy, fz) of the interpolant, then d/d(local) = * inv_vs
    const float d00 = v[1] - v[0], d10 = v[3] - v[2], d01 = v[5] - v[4], d11 = v[7] - v[6];
    const float dx0 = d00 + fy * (d10 - d00), dx1 = d01 + fy * (d11 - d01);
    const float dlx = (dx0 + fz * (dx1 - dx0)) * inv_vs;
    const float dly = ((x10 - x00) + fz * ((x11 - x01) - (x10 - x00))) * inv_vs;
    const float dlz = (y1 - y0) * inv_vs;
    // l = R p + t  =>  grad_p = R^T grad_l, R the matrix of the stored quaternion map
    const float qw = L.q.x, qx = L.q.y, qy = L.q.z, qz = L.q.w;
    const float r00 = 1.0f - 2.0f * (qy * qy + qz * qz), r01 = 2.0f * (qx * qy - qw * qz), r02 = 2.0f * (qx * qz + qw * qy);
    const float r10 = 2.0f * (qx * qy + qw * qz), r11 = 1.0f - 2.0f * (qx * qx + qz * qz), r12 = 2.0f * (qy * qz - qw * qx);
    const float r20 = 2.0f * (qx * qz - qw * qy), r21 = 2.0f * (qy * qz + qw * qx), r22 = 1.0f - 2.0f * (qx * qx + qy * qy);
    gx = r00 * dlx + r10 * dly + r20 * dlz;
    gy = r01 * dlx + r11 * dly + r21 * dlz;
    gz = r02 * dlx + r12 * dly + r22 * dlz;
    return true;
}

// Latch an error code into the model's status word (first error wins).
__device__ __forceinline__ void latch_status(int* status, int code) {
    if (status) atomicCAS(status, 0, code);
}

}  // namespace ps
