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
// 256 KiB (a single thread below that). In a process that already runs an
// OpenMP runtime under the same soname (a PyTorch process does), the team
// is that runtime's, whose threads are already up.
void stage_parallel(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPiece = 256 << 10;
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
// that ps_edge_bridge_host_inputs hands out are fixed instead (from at
// h_in, to at h_in + max_edges rows): inputs written there go over in one
// copy when n == max_edges and in two otherwise.
struct ps_edge_bridge {
    const ps_model* model = nullptr;
    ps_scene_view scene{};
    int dim = 0, max_edges = 0, device = 0;
    float *d_in = nullptr, *d_out = nullptr, *d_clr = nullptr;
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
    float *h_in = nullptr, *h_out = nullptr, *h_clr = nullptr;
    cudaStream_t stream = nullptr;
    std::list<GraphEntry> graphs;   // most recently used first
};

namespace {

void release(ps_edge_bridge* b) {
    if (!b) return;
    for (auto& g : b->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
    if (b->stream) cudaStreamDestroy(b->stream);
    cudaFree(b->d_in);
    cudaFree(b->d_out);
    cudaFree(b->d_clr);
    cudaFree(b->d_ws);
    cudaFreeHost(b->h_in);
    cudaFreeHost(b->h_out);
    cudaFreeHost(b->h_clr);
    delete b;
}

int check_edges_on(ps_edge_bridge* b, int n, const ps_edge_params* P) {
    const size_t rows = (size_t)n * b->dim;
    uint8_t* valid = reinterpret_cast<uint8_t*>(b->d_out + n);
    return ps_check_edges(b->model, &b->scene, b->d_in, b->d_in + rows, nullptr, n, P, valid, b->d_out,
                          P->compute_clearance ? b->d_clr : nullptr, b->d_ws, b->ws_bytes, b->stream);
}

// The check of n edges with these parameters on the bridge's stream: a graph
// replay when the key was seen before; otherwise an eager run, after which
// the same launches are captured for the next call with this key.
int launch_check(ps_edge_bridge* b, int n, const ps_edge_params* P) {
    GraphKey key;
    key.n = n;
    key.p = *P;
    key.v = b->scene;
    for (auto it = b->graphs.begin(); it != b->graphs.end(); ++it)
        if (it->key == key) {
            b->graphs.splice(b->graphs.begin(), b->graphs, it);
            PS_TRY_CUDA(cudaGraphLaunch(it->exec, b->stream));
            return PS_OK;
        }
    if (int rc = check_edges_on(b, n, P)) return rc;
    PS_TRY_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = check_edges_on(b, n, P);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
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
    if (b->graphs.size() >= kMaxGraphs) {
        cudaGraphExecDestroy(b->graphs.back().exec);
        b->graphs.pop_back();
    }
    b->graphs.push_front(GraphEntry{key, exec});
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
    step(cudaMalloc(&b->d_in, 2 * cfg));
    step(cudaMalloc(&b->d_out, ne * 5));
    step(cudaMalloc(&b->d_clr, ne * 4));
    step(cudaMalloc(&b->d_ws, b->ws_bytes));
    step(cudaHostAlloc(&b->h_in, 2 * cfg, cudaHostAllocDefault));
    step(cudaHostAlloc(&b->h_out, ne * 5, cudaHostAllocDefault));
    step(cudaHostAlloc(&b->h_clr, ne * 4, cudaHostAllocDefault));
    step(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
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
    *from_flat = b->h_in;
    *to_flat = b->h_in + (size_t)b->max_edges * b->dim;
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
    int dev = 0;
    PS_TRY_CUDA(cudaGetDevice(&dev));
    if (dev != b->device)
        return set_error(PS_EINVAL, "bridge created on device " + std::to_string(b->device) +
                                        ", current device is " + std::to_string(dev));
    const size_t rows = (size_t)num_edges * b->dim, bytes = rows * sizeof(float);
    float* fixed_to = b->h_in + (size_t)b->max_edges * b->dim;
    if (from_flat == b->h_in && to_flat == fixed_to) {   // written in place: nothing to stage
        if (num_edges == b->max_edges) {
            PS_TRY_CUDA(cudaMemcpyAsync(b->d_in, b->h_in, 2 * bytes, cudaMemcpyHostToDevice, b->stream));
        } else {
            PS_TRY_CUDA(cudaMemcpyAsync(b->d_in, b->h_in, bytes, cudaMemcpyHostToDevice, b->stream));
            PS_TRY_CUDA(cudaMemcpyAsync(b->d_in + rows, fixed_to, bytes, cudaMemcpyHostToDevice, b->stream));
        }
    } else {
        // Stage into the pinned mirror on OpenMP threads (one thread copies
        // 10-20 GB/s, below the host-to-device link), then copy in at once.
        stage_parallel(b->h_in, from_flat, bytes);
        stage_parallel(b->h_in + rows, to_flat, bytes);
        PS_TRY_CUDA(cudaMemcpyAsync(b->d_in, b->h_in, 2 * bytes, cudaMemcpyHostToDevice, b->stream));
    }
    if (int rc = launch_check(b, num_edges, P)) {
        cudaStreamSynchronize(b->stream);
        return rc;
    }
    const size_t n = (size_t)num_edges;
    PS_TRY_CUDA(cudaMemcpyAsync(b->h_out, b->d_out, n * 5, cudaMemcpyDeviceToHost, b->stream));
    if (P->compute_clearance)
        PS_TRY_CUDA(cudaMemcpyAsync(b->h_clr, b->d_clr, n * 4, cudaMemcpyDeviceToHost, b->stream));
    PS_TRY_CUDA(cudaStreamSynchronize(b->stream));
    std::memcpy(out_cost, b->h_out, n * 4);
    std::memcpy(out_valid, reinterpret_cast<const uint8_t*>(b->h_out + n), n);
    if (P->compute_clearance) std::memcpy(out_clearance, b->h_clr, n * 4);
    return PS_OK;
}

extern "C" int ps_edge_bridge_status(const ps_edge_bridge* b, int* status) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "bridge is NULL");
    return ps_edges_status(b->d_ws, status);
}

extern "C" int ps_edge_bridge_destroy(ps_edge_bridge* b) {
    clear_error();
    if (!b) return PS_OK;
    cudaStreamSynchronize(b->stream);
    release(b);
    return PS_OK;
}
