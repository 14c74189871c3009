// ps_stage.cuh -- shared-memory staging of the model core and the scene.
#pragma once

#include "ps_common.cuh"

namespace ps {

// Prepared record of one box from its SceneCollisionData entries: dims
// (dx, dy, dz, pad: full extents) and the inverse pose (tx, ty, tz, qw) +
// (qx, qy, qz, pad).
__device__ __forceinline__ ObbPrep prep_box(float4 dm, float4 pa, float4 pb) {
    const float qw = pa.w, qx = pb.x, qy = pb.y, qz = pb.z;
    ObbPrep p;
    // Matrix of v -> v + qw t + q x t, t = 2 q x v.
    p.r0 = make_float4(1.0f - 2.0f * (qy * qy + qz * qz), 2.0f * (qx * qy - qw * qz), 2.0f * (qx * qz + qw * qy), pa.x);
    p.r1 = make_float4(2.0f * (qx * qy + qw * qz), 1.0f - 2.0f * (qx * qx + qz * qz), 2.0f * (qy * qz - qw * qx), pa.y);
    p.r2 = make_float4(2.0f * (qx * qz - qw * qy), 2.0f * (qy * qz + qw * qx), 1.0f - 2.0f * (qx * qx + qy * qy), pa.z);
    const float hx = dm.x * 0.5f, hy = dm.y * 0.5f, hz = dm.z * 0.5f;
    const float B = fmaxf(fmaxf(fabsf(pa.x), fmaxf(fabsf(pa.y), fabsf(pa.z))), fmaxf(hx, fmaxf(hy, hz)));
    p.h = make_float4(hx, hy, hz, B);
    p.q = make_float4(qw, qx, qy, qz);
    return p;
}

// Builds the prepared box table (compacted enabled boxes, 3x3 maps, exact
// half extents) and the ESDF layer headers from the caller's
// SceneCollisionData arrays. Call with all threads; ends with __syncthreads().
// counters: 4 ints of shared scratch (slot count, stretch bound); bmax_slot:
// one float.
__device__ __forceinline__ void stage_scene(const ps_scene_view& sv, ObbPrep* obbs, int* orig, LayerPrep* layers, int* counters,
                            float* bmax_slot, SceneSmem& out) {
    if (threadIdx.x == 0) {
        counters[0] = 0;
        counters[1] = __float_as_int(1.0f);   // largest map stretch (positive floats order as ints)
        *bmax_slot = 0.0f;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < sv.n_obbs; o += blockDim.x) {
        if (sv.obb_enable[o] == 0) continue;
        const ObbPrep p = prep_box(reinterpret_cast<const float4*>(sv.obb_dims)[o],
                                   reinterpret_cast<const float4*>(sv.obb_pose)[2 * o],       // tx ty tz qw
                                   reinterpret_cast<const float4*>(sv.obb_pose)[2 * o + 1]);  // qx qy qz pad
        const float B = p.h.w;
        int slot = atomicAdd(&counters[0], 1);
        obbs[slot] = p;
        orig[slot] = o;
        atomicMax(reinterpret_cast<int*>(bmax_slot), __float_as_int(B));   // B >= 0: int order == float order
        atomicMax(&counters[1], __float_as_int(map_stretch(quat_norm_err(p.q.x, p.q.y, p.q.z, p.q.w))));
    }
    for (int l = threadIdx.x; l < sv.n_voxel_layers; l += blockDim.x) {
        LayerPrep L;
        const float4 pr = reinterpret_cast<const float4*>(sv.voxel_params)[l];
        const float4 pa = reinterpret_cast<const float4*>(sv.voxel_pose)[2 * l];
        const float4 pb = reinterpret_cast<const float4*>(sv.voxel_pose)[2 * l + 1];
        L.params = pr;
        L.enabled = (sv.voxel_enable[l] != 0) && (pr.w > 0.0f);
        const float inv_vs = pr.w > 0.0f ? __fdiv_rn(1.0f, pr.w) : 0.0f;
        L.t = make_float4(pa.x, pa.y, pa.z, inv_vs);
        L.q = make_float4(pa.w, pb.x, pb.y, pb.z);
        L.nx = robust_floor_dev(__fmul_rn(pr.x, inv_vs)) + 1;
        L.ny = robust_floor_dev(__fmul_rn(pr.y, inv_vs)) + 1;
        L.nz = robust_floor_dev(__fmul_rn(pr.z, inv_vs)) + 1;
        layers[l] = L;
        if (L.enabled) atomicMax(&counters[1], __float_as_int(map_stretch(quat_norm_err(pa.w, pb.x, pb.y, pb.z))));
    }
    __syncthreads();
    out.obbs = obbs;
    out.obb_orig = orig;
    out.layers = layers;
    out.n_obbs = counters[0];
    out.n_layers = sv.n_voxel_layers;
    out.Bmax = *bmax_slot;
    out.Mscale = __int_as_float(counters[1]);
    __syncthreads();
}

__device__ __forceinline__ uint32_t mbar_try_phase0(uint32_t bar) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar)
        : "memory");
    return done;
}

// Copies the model core (header + joint and sphere tables) into shared memory
// with one bulk async copy (cp.async.bulk, completion on an mbarrier, bounded
// wait of md.stage_polls polls). Returns false on timeout: the status is
// latched, and the copy still in flight is waited for (again bounded) so that
// it cannot land in shared memory after the block has exited. A kernel that
// gets false must write its fail-closed outputs (in collision, invalid, NaN)
// and return. Call with all threads.
__device__ __forceinline__ bool stage_model(const ModelDev& md, unsigned char* smem_blob, uint64_t* mbar) {
    const uint32_t bytes = (uint32_t)md.bytes_core;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(mbar);
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem_blob);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
            "l"(md.blob), "r"(bytes), "r"(bar)
            : "memory");
    }
    // Bounded wait on phase 0. On expiry latch PS_ETIMEOUT and give up.
    uint32_t done = 0;
    for (int it = 0; it < md.stage_polls && !done; ++it) done = mbar_try_phase0(bar);
    int ok = __syncthreads_and((int)done);
    if (!ok) {
        if (threadIdx.x == 0) latch_status(md.status, PS_ETIMEOUT);
        // drain: the copy may still be in flight (bounded as well)
        uint32_t landed = done;
        for (int it = 0; it < PS_STAGE_POLLS && !landed; ++it) landed = mbar_try_phase0(bar);
        __syncthreads();
    }
    return ok != 0;
}

}  // namespace ps
