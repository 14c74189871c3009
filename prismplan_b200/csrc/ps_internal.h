// ps_internal.h -- host-side internals shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ps_common.cuh"

// Host handle behind the opaque ps_model*.
struct ps_model {
    ps::ModelDev dev{};
    void* alloc = nullptr;      // single device allocation
    size_t alloc_bytes = 0;
    ps_model_info info{};
    int max_joint_spheres = 0;  // most exact spheres on one joint
    bool root_slot_only = false; // slot 0 holds only the root (identity) frame
    int max_joint_approx = 0;
    std::vector<int> sph_orig;  // reordered -> descriptor index (host copy)
};

#include <nvtx3/nvToolsExt.h>

namespace ps {

// NVTX range around a C-ABI call (profilers show each call by name; a no-op
// when no tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define PS_NVTX(name) ::ps::NvtxRange ps_nvtx_range_(name)

int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* where);
void clear_error();

// Trajectory cost launcher behind ps_traj_cost (same arguments, stream
// typed). skip (device [B] or NULL): trajectories b with skip[b] != 0 need
// no output (the batched optimisers skip finished requests this way); their
// outputs may still be written, with the values an unskipped launch writes.
int traj_cost_launch(const ps_model* m, const ps_scene_view* scene, const float* q, int B, int T,
                     const ps_cost_params* P, float* waypoint_cost, float* traj_cost, float* grad,
                     const uint8_t* skip, cudaStream_t s);

// Validate a scene view against a model (and the model's device, below);
// returns PS_OK or sets the error.
int validate_scene(const ps_model* m, const ps_scene_view* s);
// The model's blob lives on the device it was created on: PS_EINVAL (with a
// message) unless that device is the current one. Every kernel reads the
// blob, so running with another device current would read another GPU's
// memory.
int check_model_device(const ps_model* m);

// Dynamic shared memory needed to stage model core + scene tables.
size_t scene_smem_bytes(const ps_scene_view* s);

// Opts `func` into `bytes` of dynamic shared memory on the current device
// (cudaFuncSetAttribute), remembering the largest amount set per device and
// kernel so that repeated launches skip the call.
cudaError_t allow_smem(const void* func, size_t bytes);

// Number of SMs of the current device (cached).
int sm_count();
// Largest dynamic shared memory one block may opt into on the current device.
size_t smem_optin();

// Diagnostics shared by every launcher (set through ps_set_stats /
// ps_set_timing_events).
extern unsigned long long* g_stats;
extern cudaEvent_t g_ev_start, g_ev_stop;
// Inside a stream capture a plain cudaEventRecord only expresses a
// dependency; an external record node is what re-records on every replay.
inline void mark_event(cudaEvent_t e, cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &st);
    if (st == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else cudaEventRecord(e, s);
}
inline void mark_start(cudaStream_t s) {
    if (g_ev_start && g_ev_stop) mark_event(g_ev_start, s);
}
inline void mark_stop(cudaStream_t s) {
    if (g_ev_start && g_ev_stop) mark_event(g_ev_stop, s);
}

}  // namespace ps

#define PS_TRY_CUDA(expr)                                        \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return ps::cuda_error(_e, #expr); \
    } while (0)
