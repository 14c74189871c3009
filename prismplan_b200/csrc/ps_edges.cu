// ps_edges.cu -- edge checks: plain (one warp per edge) and persistent
// (chunk-major global work queue, capture-safe).
//
// Replaces evaluate_edges_batch + EdgeEvalGpu::evaluate
// (code/gpu_planning/cpp/src/planning/edge_eval.cuh:64-165,
// edge_batch_bridge.hh:60-96). Per edge the verdict is the OR over samples
// j = 1..G (t = j/G, interpolated as from + t*(to - from) with one rounding of
// the product-sum) of the two-phase verdict, exactly as the reference forms it;
// cost = sqrtf(sum d*d) if valid, else FLT_MAX.
//
// Warp layout: a warp owns one chunk of 32 consecutive samples of one edge,
// lane = sample. Samples of a chunk are close in configuration space, so per
// joint the warp first bounds the 32 link positions by one sphere and culls
// the boxes it cannot reach (a conservative broad phase with the same guard
// band as the pair path), then runs the gate and exact tests against the
// survivors only; an __any_sync after every joint retires the chunk (and the
// edge) at the first confirmed hit. With enough edges to fill the GPU, an
// end-sample probe (one thread per edge, sample j = G) runs first and retires
// the edges that collide there before the queue starts.
#include <algorithm>
#include <cfloat>
#include <mutex>
#include <string>
#include <vector>

#include "ps_edgekern.cuh"

using namespace ps;

namespace {

int check_edge_args(const ps_model* m, const ps_scene_view* scene, const float* from, const float* to, int n,
                    const ps_edge_params* P, uint8_t* valid, float* cost) {
    if (!m) return set_error(PS_EINVAL, "model is NULL");
    if (!P) return set_error(PS_EINVAL, "params is NULL");
    if (n < 0) return set_error(PS_EINVAL, "n_edges < 0");
    if (n > 0 && (!from || !to || !valid || !cost)) return set_error(PS_EINVAL, "from/to/valid/cost NULL");
    if (P->max_samples > 0 && P->max_samples > (1 << 20))
        return set_error(PS_EINVAL, "max_samples above 2^20");
    if (P->probe < 0 || P->probe > 2 || P->queue_blocks_per_sm < 0 || P->grab < 0 || P->grab > 32)
        return set_error(PS_EINVAL, "probe must be 0..2, queue_blocks_per_sm >= 0, grab 0..32");
    return validate_scene(m, scene);
}

}  // namespace

extern "C" int ps_check_edges_plain(const ps_model* m, const ps_scene_view* scene, const float* from,
                                    const float* to, const int* samples_per_edge, int n_edges,
                                    const ps_edge_params* P, uint8_t* valid, float* cost, float* clearance,
                                    void* stream) {
    PS_NVTX("ps_check_edges_plain");
    clear_error();
    if (int rc = check_edge_args(m, scene, from, to, n_edges, P, valid, cost)) return rc;
    if (n_edges == 0) return PS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t smem = edge_smem_bytes(m, scene);
    const int grid = (n_edges + kWarps - 1) / kWarps;
    auto kern = pick(fast_path(m, scene, P), g_stats != nullptr, edges_plain_kernel<0, false>,
                     edges_plain_kernel<0, true>, edges_plain_kernel<1, false>, edges_plain_kernel<1, true>,
                     edges_plain_kernel<2, false>, edges_plain_kernel<2, true>);
    PS_TRY_CUDA(allow_smem((const void*)kern, smem));
    mark_start(s);
    kern<<<grid, kEdgeThreads, smem, s>>>(m->dev, *scene, *P, from, to, samples_per_edge, n_edges, valid, cost,
                                          clearance, g_stats);
    mark_stop(s);
    PS_TRY_CUDA(cudaGetLastError());
    return launch_edges_self(m, P, from, to, samples_per_edge, n_edges, nullptr, nullptr, valid, cost, nullptr,
                             nullptr, s);
}

extern "C" size_t ps_edges_workspace_bytes(int n_edges) {
    const size_t n = (size_t)std::max(n_edges, 1);
    return align256(sizeof(EdgeWs)) + 6 * align256(n * 4);
}

namespace {

// Workspace layout: header, then per-edge G, length, retire flag,
// ordered-int clearance, completed-chunk count and the long list (the edges
// with more than one chunk round), 4 B each.
struct EdgeBufs {
    EdgeWs* hdr;
    int *G, *bad, *clr, *done, *lst;
    float* len;
};

EdgeBufs carve_workspace(void* ws, int n_edges) {
    unsigned char* w = reinterpret_cast<unsigned char*>(ws);
    const size_t seg = align256((size_t)n_edges * 4);
    EdgeBufs b;
    b.hdr = reinterpret_cast<EdgeWs*>(w);
    unsigned char* p = w + align256(sizeof(EdgeWs));
    b.G = reinterpret_cast<int*>(p);
    b.len = reinterpret_cast<float*>(p + seg);
    b.bad = reinterpret_cast<int*>(p + 2 * seg);
    b.clr = reinterpret_cast<int*>(p + 3 * seg);
    b.done = reinterpret_cast<int*>(p + 4 * seg);
    b.lst = reinterpret_cast<int*>(p + 5 * seg);
    return b;
}

// memset header -> prep -> end-sample probe -> queue pass(es) -> self pass ->
// finalize on stream s.
int run_persistent(const ps_model* m, const ps_scene_view* scene, const float* from, const float* to,
                   const int* samples_per_edge, int n_edges, const ps_edge_params* P, uint8_t* valid, float* cost,
                   float* clearance, const EdgeBufs& b, cudaStream_t s) {
    const int D = m->info.n_dof;
    PS_TRY_CUDA(cudaMemsetAsync(b.hdr, 0, sizeof(EdgeWs), s));   // queue heads, deadline, max rounds, timeout
    const size_t smem = edge_smem_bytes(m, scene);
    const int mode = fast_path(m, scene, P);
    auto qk = pick(mode, g_stats != nullptr, edges_queue_kernel<0, false>, edges_queue_kernel<0, true>,
                   edges_queue_kernel<1, false>, edges_queue_kernel<1, true>, edges_queue_kernel<2, false>,
                   edges_queue_kernel<2, true>);
    PS_TRY_CUDA(allow_smem((const void*)qk, smem));
    int per_sm = 0;
    PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qk, kEdgeThreads, smem));
    per_sm = std::max(per_sm, 1);
    if (P->queue_blocks_per_sm > 0) per_sm = std::min(per_sm, P->queue_blocks_per_sm);
    const int qgrid = std::max(1, sm_count() * per_sm);
    // With few edges per resident warp the queue runs round 0 in a pass of its
    // own; the second pass then visits only the edges listed as having more
    // rounds (a CHOMP loop's 16 K short segments: 34.7 -> 29.9 ms per call).
    // With many, one pass runs every round over every edge, as before.
    const bool split = (long long)n_edges < 8ll * qgrid * kEdgeThreads / 32;   // the kernel's own split rule
    int* lst = split ? b.lst : nullptr;
    ProbePlan probe;
    if (int rc = plan_probe(m, scene, mode, g_stats != nullptr, 1.0f, n_edges, P->probe, probe)) return rc;
    if (!probe.kp) {   // with the probe, its launch also prepares the edges
        const int pgrid = std::max(1, std::min((n_edges + 255) / 256, sm_count() * 4));
        edges_prep_kernel<<<pgrid, 256, 0, s>>>(*P, from, to, samples_per_edge, n_edges, D, b.hdr, b.G, b.len, b.bad,
                                                b.clr, b.done, nullptr, lst);
        PS_TRY_CUDA(cudaGetLastError());
    }
    mark_start(s);
    if (probe.kp)
        probe.kp<<<probe.grid, kProbeThreads, probe.smem, s>>>(m->dev, *scene, *P, from, to, n_edges, b.hdr, b.G,
                                                                b.bad, g_stats, nullptr,
                                                                PrepArgs{samples_per_edge, b.len, b.clr, b.done, lst});
    qk<<<qgrid, kEdgeThreads, smem, s>>>(m->dev, *scene, *P, from, to, n_edges, b.hdr, b.G, b.bad, b.clr, b.done,
                                         g_stats, 0, nullptr, lst);
    if (split)
        qk<<<qgrid, kEdgeThreads, smem, s>>>(m->dev, *scene, *P, from, to, n_edges, b.hdr, b.G, b.bad, b.clr, b.done,
                                             g_stats, 1, nullptr, lst);
    mark_stop(s);
    PS_TRY_CUDA(cudaGetLastError());
    if (int rc = launch_edges_self(m, P, from, to, samples_per_edge, n_edges, b.G, b.bad, nullptr, nullptr, b.hdr,
                                   nullptr, s))
        return rc;
    const int fgrid = std::max(1, std::min((n_edges + 255) / 256, sm_count() * 4));
    edges_finalize_kernel<<<fgrid, 256, 0, s>>>(n_edges, *P, b.bad, b.len, b.clr, b.done, b.G, b.hdr, valid, cost,
                                                clearance);
    PS_TRY_CUDA(cudaGetLastError());
    return PS_OK;
}

}  // namespace

extern "C" int ps_check_edges(const ps_model* m, const ps_scene_view* scene, const float* from, const float* to,
                              const int* samples_per_edge, int n_edges, const ps_edge_params* P, uint8_t* valid,
                              float* cost, float* clearance, void* workspace, size_t workspace_bytes, void* stream) {
    PS_NVTX("ps_check_edges");
    clear_error();
    if (int rc = check_edge_args(m, scene, from, to, n_edges, P, valid, cost)) return rc;
    if (n_edges == 0) return PS_OK;
    if (!workspace || workspace_bytes < ps_edges_workspace_bytes(n_edges))
        return set_error(PS_EINVAL, "workspace missing or smaller than ps_edges_workspace_bytes(n_edges)");
    if ((reinterpret_cast<uintptr_t>(workspace) & 15) != 0) return set_error(PS_EINVAL, "workspace not 16-byte aligned");
    return run_persistent(m, scene, from, to, samples_per_edge, n_edges, P, valid, cost, clearance,
                          carve_workspace(workspace, n_edges), (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Edge checks without a caller-provided workspace.
//
// Some callers cannot hand the library a device allocation: a planner that
// evaluates an edge batch per search expansion inside a latency budget cannot
// afford cudaMalloc / cudaFree (they can synchronise the whole device), and
// some host processes have no CUDA allocator of their own to draw from (a
// plugin loaded into a framework that owns all device memory, or a
// fixed-memory real-time process). For them the persistent path's workspace
// lives in the library itself: a file-scope device array sized for
// PS_EDGES_STATIC_MAX edges, which every GPU that loads the library holds
// until the process exits. Nothing here allocates.
//
// The array is shared by every call: a call resets what must start at zero
// (queue head and max G) and its prep kernel rewrites the per-edge state, so
// back-to-back calls are fine, but calls whose kernels overlap on the GPU
// (other streams, other host threads) race on it.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kStaticWsBytes =
    ((sizeof(EdgeWs) + 255) & ~size_t(255)) + 6 * (((size_t)PS_EDGES_STATIC_MAX * 4 + 255) & ~size_t(255));

static __device__ __align__(256) unsigned char g_edges_static_ws[kStaticWsBytes];

// Device address of g_edges_static_ws per device ordinal (host code must not
// use the symbol itself: on the host it only names a stand-in).
std::mutex g_static_ws_mutex;
void* g_static_ws_ptr[128] = {nullptr};

int static_workspace(void** out) {
    int dev = 0;
    PS_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return set_error(PS_EINVAL, "device ordinal above 127");
    std::lock_guard<std::mutex> lock(g_static_ws_mutex);
    if (!g_static_ws_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_edges_static_ws);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_edges_static_ws)");
        g_static_ws_ptr[dev] = p;
    }
    *out = g_static_ws_ptr[dev];
    return PS_OK;
}

}  // namespace

extern "C" int ps_check_edges_static(const ps_model* m, const ps_scene_view* scene, const float* from,
                                     const float* to, const int* samples_per_edge, int n_edges,
                                     const ps_edge_params* P, uint8_t* valid, float* cost, float* clearance,
                                     void* stream) {
    PS_NVTX("ps_check_edges_static");
    clear_error();
    if (int rc = check_edge_args(m, scene, from, to, n_edges, P, valid, cost)) return rc;
    if (n_edges > PS_EDGES_STATIC_MAX)
        return set_error(PS_EINVAL, "n_edges " + std::to_string(n_edges) + " exceeds the built-in workspace (" +
                                        std::to_string(PS_EDGES_STATIC_MAX) +
                                        " edges); split the batch or use ps_check_edges with a workspace");
    if (n_edges == 0) return PS_OK;
    void* ws = nullptr;
    if (int rc = static_workspace(&ws)) return rc;
    return run_persistent(m, scene, from, to, samples_per_edge, n_edges, P, valid, cost, clearance,
                          carve_workspace(ws, n_edges), (cudaStream_t)stream);
}

extern "C" int ps_edges_status(const void* workspace, int* status) {
    clear_error();
    if (!status) return set_error(PS_EINVAL, "status is NULL");
    void* ws = const_cast<void*>(workspace);
    if (!ws)
        if (int rc = static_workspace(&ws)) return rc;
    EdgeWs h;
    PS_TRY_CUDA(cudaMemcpy(&h, ws, sizeof(EdgeWs), cudaMemcpyDeviceToHost));
    *status = h.timed_out ? PS_ETIMEOUT : PS_OK;
    return PS_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the persistent path's launch shape.
// ---------------------------------------------------------------------------
namespace {

// Median time (ms) of `reps` calls of fn on stream s, after one untimed call.
template <class F>
int time_calls(F fn, cudaStream_t s, int reps, float& ms_out) {
    cudaEvent_t a = nullptr, z = nullptr;
    PS_TRY_CUDA(cudaEventCreate(&a));
    if (cudaEventCreate(&z) != cudaSuccess) {
        cudaEventDestroy(a);
        return cuda_error(cudaGetLastError(), "tuning events");
    }
    int rc = fn();
    std::vector<float> ms;
    for (int r = 0; r < reps && rc == PS_OK; ++r) {
        cudaEventRecord(a, s);
        rc = fn();
        cudaEventRecord(z, s);
        if (rc == PS_OK && cudaEventSynchronize(z) != cudaSuccess) rc = cuda_error(cudaGetLastError(), "tuning run");
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, z);
        ms.push_back(t);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    if (rc) return rc;
    std::sort(ms.begin(), ms.end());
    ms_out = ms[ms.size() / 2];
    return PS_OK;
}

}  // namespace

extern "C" int ps_tune_edges(const ps_model* m, const ps_scene_view* scene, const float* from, const float* to,
                             const int* samples_per_edge, int n_edges, const ps_edge_params* P, uint8_t* valid,
                             float* cost, float* clearance, void* workspace, size_t workspace_bytes, void* stream,
                             ps_edge_tuning* out, ps_edge_params* tuned) {
    PS_NVTX("ps_tune_edges");
    clear_error();
    if (!P || !tuned) return set_error(PS_EINVAL, "params / tuned is NULL");
    if (int rc = check_edge_args(m, scene, from, to, n_edges, P, valid, cost)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    ps_edge_params p = *P;
    auto run = [&]() {
        return ps_check_edges(m, scene, from, to, samples_per_edge, n_edges, &p, valid, cost, clearance, workspace,
                              workspace_bytes, stream);
    };
    p.probe = p.queue_blocks_per_sm = p.grab = 0;
    float def_ms = 0.0f;
    if (int rc = time_calls(run, s, 5, def_ms)) return rc;
    // candidates: probe on/off (on only where the probe exists), the queue's
    // residency from all that fit down by two, three grab sizes
    const int mode = fast_path(m, scene, P);
    int per_sm = 0;
    {
        const size_t smem = edge_smem_bytes(m, scene);
        auto qk = pick(mode, false, edges_queue_kernel<0, false>, edges_queue_kernel<0, true>,
                       edges_queue_kernel<1, false>, edges_queue_kernel<1, true>, edges_queue_kernel<2, false>,
                       edges_queue_kernel<2, true>);
        PS_TRY_CUDA(allow_smem((const void*)qk, smem));
        PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qk, kEdgeThreads, smem));
        per_sm = std::max(per_sm, 1);
    }
    std::vector<int> probes = {2};
    if (mode == 1 && scene->n_obbs > 0) probes.push_back(1);
    float best = def_ms;
    ps_edge_params best_p = p;
    int n_cand = 1;
    for (int pr : probes)
        for (int q = per_sm; q >= std::max(1, per_sm - 2); --q)
            for (int g : {0, 8, 32}) {
                p.probe = pr;
                p.queue_blocks_per_sm = q;
                p.grab = g;
                float ms = 0.0f;
                if (int rc = time_calls(run, s, 3, ms)) return rc;
                ++n_cand;
                if (ms < best) {
                    best = ms;
                    best_p = p;
                }
            }
    *tuned = *P;
    tuned->probe = best_p.probe;
    tuned->queue_blocks_per_sm = best_p.queue_blocks_per_sm;
    tuned->grab = best_p.grab;
    if (out) *out = ps_edge_tuning{best_p.probe, best_p.queue_blocks_per_sm, best_p.grab, best, def_ms, n_cand};
    return PS_OK;
}
