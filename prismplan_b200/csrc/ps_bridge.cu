// ps_bridge.cu -- host-buffer edge bridge: the C-ABI counterpart of
// ppln::search::EdgeEvalGpu (code/gpu_planning/cpp/src/planning/
// edge_batch_bridge.hh:27-111).
//
// Like the reference class it owns device buffers sized for max_edges, pinned
// host mirrors and a private stream, and evaluate() takes host arrays, copies
// them in, checks, copies the outputs back and synchronises. Three things
// differ, none of them in the results:
//   * the check is the persistent edge path (ps_check_edges), replayed from a
//     CUDA graph per (edge count, parameters, scene) instead of re-issued;
//   * the host-side staging into the pinned mirrors runs on OpenMP threads
//     (the reference copies with one thread), and a caller that writes its
//     edges straight into the mirrors (ps_edge_bridge_host_inputs) skips it;
//   * status codes instead of exceptions (the reference throws on
//     num_edges > max_edges, :67-68; here PS_EINVAL).
#include <algorithm>
#include <cstring>
#include <list>
#include <string>
#include <vector>

#include <omp.h>

#include "ps_internal.h"

using namespace ps;

namespace {

constexpr size_t kMaxGraphs = 8;

// Host copy of `bytes` split over OpenMP threads in pieces of at least
// 128 KiB (a single thread below that). In a process that already runs an
// OpenMP runtime under the same soname (a PyTorch process does), the team
// is that runtime's, whose threads are already up.
void stage_parallel(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPiece = 128 << 10;
    const int pieces = (int)std::min<size_t>((bytes + kPiece - 1) / kPiece, 64);
    const int threads = std::min(pieces, std::max(1, omp_get_max_threads()));
    if (threads <= 1) {
        std::memmove(dst, src, bytes);
        return;
    }
    const size_t step = (bytes / (size_t)pieces + 63) & ~size_t(63);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int k = 0; k < pieces; ++k) {
        const size_t lo = (size_t)k * step;
        if (lo < bytes)
            std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, std::min(step, bytes - lo));
    }
}

bool same_view(const ps_scene_view& a, const ps_scene_view& b) {
    return a.obb_dims == b.obb_dims && a.obb_pose == b.obb_pose && a.obb_enable == b.obb_enable &&
           a.n_obbs == b.n_obbs && a.voxel_params == b.voxel_params && a.voxel_pose == b.voxel_pose &&
           a.voxel_enable == b.voxel_enable && a.voxel_features == b.voxel_features &&
           a.n_voxel_layers == b.n_voxel_layers && a.max_voxels_per_layer == b.max_voxels_per_layer &&
           a.sphere_acm_mask == b.sphere_acm_mask && a.sphere_obb_acm_mask == b.sphere_obb_acm_mask &&
           a.sphere_obb_acm_mask_approx == b.sphere_obb_acm_mask_approx && a.esdf_mode == b.esdf_mode;
}

struct GraphKey {
    int n;
    ps_edge_params p;
    ps_scene_view v;
    bool operator==(const GraphKey& o) const {
        return n == o.n && std::memcmp(&p, &o.p, sizeof(p)) == 0 && same_view(v, o.v);   // p: 4-byte fields only
    }
};

struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

// Buffers are packed per call so that each direction is one copy: for n
// edges the device inputs are d_in = [from (n rows) | to (n rows)] and the
// device outputs d_out = [cost (n floats) | valid (n bytes)]; the pinned
// mirrors h_in and h_out hold the same layouts. The in-place input mirrors
// that ps_edge_bridge_host_inputs hands out (slot 0's) are fixed instead
// (from at h_in, to at h_in + max_edges rows): inputs written there go over
// in one copy when n == max_edges and in two otherwise.
//
// A slot holds one call in flight: its buffers, workspace, stream, captured
// graphs and a completion event. Two slots let a caller stage and copy in
// one batch while the GPU checks the other.
struct BridgeSlot {
    float *d_in = nullptr, *d_out = nullptr, *d_clr = nullptr;
    void* d_ws = nullptr;
    float *h_in = nullptr, *h_out = nullptr, *h_clr = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::list<GraphEntry> graphs;   // most recently used first
    bool pending = false;           // submitted, not yet waited for
    int n = 0;
    bool clearance = false;
};

struct ps_edge_bridge {
    const ps_model* model = nullptr;
    ps_scene_view scene{};
    int dim = 0, max_edges = 0, device = 0;
    size_t ws_bytes = 0;
    BridgeSlot slot[PS_BRIDGE_SLOTS];
    int last_slot = 0;   // slot of the last call waited for
};

namespace {

void release_slot(BridgeSlot& sl) {
    for (auto& g : sl.graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    sl.graphs.clear();
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    cudaFree(sl.d_in);
    cudaFree(sl.d_out);
    cudaFree(sl.d_clr);
    cudaFree(sl.d_ws);
    cudaFreeHost(sl.h_in);
    cudaFreeHost(sl.h_out);
    cudaFreeHost(sl.h_clr);
}

void release(ps_edge_bridge* b) {
    if (!b) return;
    for (auto& sl : b->slot) release_slot(sl);
    delete b;
}

int check_edges_on(ps_edge_bridge* b, BridgeSlot& sl, int n, const ps_edge_params* P) {
    const size_t rows = (size_t)n * b->dim;
    uint8_t* valid = reinterpret_cast<uint8_t*>(sl.d_out + n);
    return ps_check_edges(b->model, &b->scene, sl.d_in, sl.d_in + rows, nullptr, n, P, valid, sl.d_out,
                          P->compute_clearance ? sl.d_clr : nullptr, sl.d_ws, b->ws_bytes, sl.stream);
}

// The check of n edges with these parameters on the slot's stream: a graph
// replay when the key was seen before; otherwise an eager run, after which
// the same launches are captured for the next call with this key.
int launch_check(ps_edge_bridge* b, BridgeSlot& sl, int n, const ps_edge_params* P) {
    GraphKey key;
    key.n = n;
    key.p = *P;
    key.v = b->scene;
    for (auto it = sl.graphs.begin(); it != sl.graphs.end(); ++it)
        if (it->key == key) {
            sl.graphs.splice(sl.graphs.begin(), sl.graphs, it);
            PS_TRY_CUDA(cudaGraphLaunch(it->exec, sl.stream));
            return PS_OK;
        }
    if (int rc = check_edges_on(b, sl, n, P)) return rc;
    PS_TRY_CUDA(cudaStreamBeginCapture(sl.stream, cudaStreamCaptureModeThreadLocal));
    const int rc = check_edges_on(b, sl, n, P);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(sl.stream, &g);
    if (rc != PS_OK || e != cudaSuccess || !g) {   // not kept: the eager run above already did the work
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return PS_OK;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        cudaGetLastError();
        return PS_OK;
    }
    if (sl.graphs.size() >= kMaxGraphs) {
        cudaGraphExecDestroy(sl.graphs.back().exec);
        sl.graphs.pop_back();
    }
    sl.graphs.push_front(GraphEntry{key, exec});
    return PS_OK;
}

int check_slot_arg(const ps_edge_bridge* b, int slot) {
    if (!b) return set_error(PS_EINVAL, "bridge is NULL");
    if (slot < 0 || slot >= PS_BRIDGE_SLOTS)
        return set_error(PS_EINVAL, "slot must be 0 .. " + std::to_string(PS_BRIDGE_SLOTS - 1));
    int dev = 0;
    PS_TRY_CUDA(cudaGetDevice(&dev));
    if (dev != b->device)
        return set_error(PS_EINVAL, "bridge created on device " + std::to_string(b->device) +
                                        ", current device is " + std::to_string(dev));
    return PS_OK;
}

}  // namespace

extern "C" int ps_edge_bridge_create(const ps_model* model, const ps_scene_view* scene, int dim, int max_edges,
                                     ps_edge_bridge** out) {
    PS_NVTX("ps_edge_bridge_create");
    clear_error();
    if (!out) return set_error(PS_EINVAL, "out is NULL");
    *out = nullptr;
    if (!model) return set_error(PS_EINVAL, "model is NULL");
    if (dim != model->info.n_dof)
        return set_error(PS_EINVAL, "dim " + std::to_string(dim) + " differs from the model's n_dof " +
                                        std::to_string(model->info.n_dof));
    if (max_edges <= 0) return set_error(PS_EINVAL, "max_edges must be > 0");
    if (int rc = validate_scene(model, scene)) return rc;
    auto* b = new ps_edge_bridge();
    b->model = model;
    b->scene = *scene;
    b->dim = dim;
    b->max_edges = max_edges;
    cudaGetDevice(&b->device);
    const size_t cfg = (size_t)max_edges * dim * sizeof(float);
    const size_t ne = (size_t)max_edges;
    b->ws_bytes = ps_edges_workspace_bytes(max_edges);
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    for (auto& sl : b->slot) {
        step(cudaMalloc(&sl.d_in, 2 * cfg));
        step(cudaMalloc(&sl.d_out, ne * 5));
        step(cudaMalloc(&sl.d_clr, ne * 4));
        step(cudaMalloc(&sl.d_ws, b->ws_bytes));
        step(cudaHostAlloc(&sl.h_in, 2 * cfg, cudaHostAllocDefault));
        step(cudaHostAlloc(&sl.h_out, ne * 5, cudaHostAllocDefault));
        step(cudaHostAlloc(&sl.h_clr, ne * 4, cudaHostAllocDefault));
        step(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
        step(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    }
    if (e != cudaSuccess) {
        release(b);
        return cuda_error(e, "ps_edge_bridge_create allocations");
    }
    *out = b;
    return PS_OK;
}

extern "C" int ps_edge_bridge_set_scene(ps_edge_bridge* b, const ps_scene_view* scene) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "bridge is NULL");
    if (int rc = validate_scene(b->model, scene)) return rc;
    b->scene = *scene;
    return PS_OK;
}

extern "C" int ps_edge_bridge_host_inputs(ps_edge_bridge* b, float** from_flat, float** to_flat) {
    clear_error();
    if (!b || !from_flat || !to_flat) return set_error(PS_EINVAL, "bridge or output pointer is NULL");
    *from_flat = b->slot[0].h_in;
    *to_flat = b->slot[0].h_in + (size_t)b->max_edges * b->dim;
    return PS_OK;
}

extern "C" int ps_edge_bridge_submit(ps_edge_bridge* b, int slot, const float* from_flat, const float* to_flat,
                                     int num_edges, const ps_edge_params* P) {
    PS_NVTX("ps_edge_bridge_submit");
    clear_error();
    if (int rc = check_slot_arg(b, slot)) return rc;
    if (!P) return set_error(PS_EINVAL, "params is NULL");
    BridgeSlot& sl = b->slot[slot];
    if (sl.pending) return set_error(PS_EINVAL, "slot " + std::to_string(slot) + " has a call not yet waited for");
    if (num_edges > b->max_edges)
        return set_error(PS_EINVAL, "num_edges " + std::to_string(num_edges) + " exceeds max_edges " +
                                        std::to_string(b->max_edges));
    sl.n = num_edges > 0 ? num_edges : 0;
    sl.clearance = P->compute_clearance != 0;
    if (sl.n == 0) {   // the reference returns empty outputs (:66)
        sl.pending = true;
        return PS_OK;
    }
    if (!from_flat || !to_flat) return set_error(PS_EINVAL, "from_flat/to_flat NULL");
    const size_t rows = (size_t)num_edges * b->dim, bytes = rows * sizeof(float);
    float* fixed_to = sl.h_in + (size_t)b->max_edges * b->dim;
    if (from_flat == sl.h_in && to_flat == fixed_to) {   // written in place: nothing to stage
        if (num_edges == b->max_edges) {
            PS_TRY_CUDA(cudaMemcpyAsync(sl.d_in, sl.h_in, 2 * bytes, cudaMemcpyHostToDevice, sl.stream));
        } else {
            PS_TRY_CUDA(cudaMemcpyAsync(sl.d_in, sl.h_in, bytes, cudaMemcpyHostToDevice, sl.stream));
            PS_TRY_CUDA(cudaMemcpyAsync(sl.d_in + rows, fixed_to, bytes, cudaMemcpyHostToDevice, sl.stream));
        }
    } else {
        // Stage into the pinned mirror on OpenMP threads (one thread copies
        // 10-20 GB/s, below the host-to-device link): the `from` rows first,
        // whose copy in then runs while the `to` rows are staged. The slot's
        // previous call was waited for, so its mirror is free.
        stage_parallel(sl.h_in, from_flat, bytes);
        PS_TRY_CUDA(cudaMemcpyAsync(sl.d_in, sl.h_in, bytes, cudaMemcpyHostToDevice, sl.stream));
        stage_parallel(sl.h_in + rows, to_flat, bytes);
        PS_TRY_CUDA(cudaMemcpyAsync(sl.d_in + rows, sl.h_in + rows, bytes, cudaMemcpyHostToDevice, sl.stream));
    }
    if (int rc = launch_check(b, sl, num_edges, P)) {
        cudaStreamSynchronize(sl.stream);
        return rc;
    }
    const size_t n = (size_t)num_edges;
    PS_TRY_CUDA(cudaMemcpyAsync(sl.h_out, sl.d_out, n * 5, cudaMemcpyDeviceToHost, sl.stream));
    if (sl.clearance) PS_TRY_CUDA(cudaMemcpyAsync(sl.h_clr, sl.d_clr, n * 4, cudaMemcpyDeviceToHost, sl.stream));
    PS_TRY_CUDA(cudaEventRecord(sl.done, sl.stream));
    sl.pending = true;
    return PS_OK;
}

extern "C" int ps_edge_bridge_wait(ps_edge_bridge* b, int slot, uint8_t* out_valid, float* out_cost,
                                   float* out_clearance) {
    PS_NVTX("ps_edge_bridge_wait");
    clear_error();
    if (int rc = check_slot_arg(b, slot)) return rc;
    BridgeSlot& sl = b->slot[slot];
    if (!sl.pending) return set_error(PS_EINVAL, "slot " + std::to_string(slot) + " has no call to wait for");
    const size_t n = (size_t)sl.n;
    if (n > 0 && (!out_valid || !out_cost)) return set_error(PS_EINVAL, "out_valid/out_cost NULL");
    if (n > 0 && sl.clearance && !out_clearance)
        return set_error(PS_EINVAL, "compute_clearance was set but out_clearance is NULL");
    sl.pending = false;
    if (n == 0) return PS_OK;
    PS_TRY_CUDA(cudaEventSynchronize(sl.done));
    std::memcpy(out_cost, sl.h_out, n * 4);
    std::memcpy(out_valid, reinterpret_cast<const uint8_t*>(sl.h_out + n), n);
    if (sl.clearance) std::memcpy(out_clearance, sl.h_clr, n * 4);
    b->last_slot = slot;
    return PS_OK;
}

extern "C" int ps_edge_bridge_evaluate(ps_edge_bridge* b, const float* from_flat, const float* to_flat,
                                       int num_edges, const ps_edge_params* P, uint8_t* out_valid,
                                       float* out_cost, float* out_clearance) {
    PS_NVTX("ps_edge_bridge_evaluate");
    clear_error();
    if (!b) return set_error(PS_EINVAL, "bridge is NULL");
    if (!P) return set_error(PS_EINVAL, "params is NULL");
    if (num_edges <= 0) return PS_OK;   // the reference returns empty outputs (:66)
    if (num_edges > b->max_edges)
        return set_error(PS_EINVAL, "num_edges " + std::to_string(num_edges) + " exceeds max_edges " +
                                        std::to_string(b->max_edges));
    if (!from_flat || !to_flat || !out_valid || !out_cost)
        return set_error(PS_EINVAL, "from_flat/to_flat/out_valid/out_cost NULL");
    if (P->compute_clearance && !out_clearance)
        return set_error(PS_EINVAL, "compute_clearance set but out_clearance is NULL");
    if (b->slot[0].pending) return set_error(PS_EINVAL, "slot 0 has a submitted call not yet waited for");
    if (int rc = ps_edge_bridge_submit(b, 0, from_flat, to_flat, num_edges, P)) {
        b->slot[0].pending = false;
        return rc;
    }
    return ps_edge_bridge_wait(b, 0, out_valid, out_cost, out_clearance);
}

extern "C" int ps_edge_bridge_status(const ps_edge_bridge* b, int* status) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "bridge is NULL");
    return ps_edges_status(b->slot[b->last_slot].d_ws, status);
}

extern "C" int ps_edge_bridge_destroy(ps_edge_bridge* b) {
    clear_error();
    if (!b) return PS_OK;
    for (auto& sl : b->slot)
        if (sl.stream) cudaStreamSynchronize(sl.stream);
    release(b);
    return PS_OK;
}
