// ps_batch.cu -- mixed-request batches: many edge-check requests of uneven
// length and many trajectory cost+gradient requests in one CUDA-graph launch.
//
// The reference evaluates each request with its own launches and a host sync
// (EdgeEvalGpu::evaluate, edge_batch_bridge.hh:60-96; the CHOMP loop,
// chomp.cu:508-555; STOMP's state cost launch, stomp.cu:206-245). Here a batch
// keeps its request table in pinned host memory and one captured graph
//   1. copies the table and the live counts to the device,
//   2. forks two branches that run concurrently on disjoint SM shares:
//      edges:        gather rows + resolve G -> prep -> persistent chunk-major
//                    queue kernel -> finalize -> scatter to each request;
//      trajectories: gather waypoints -> one cost+adjoint kernel over every
//                    waypoint -> one block per request adds the smoothness
//                    term and writes the request's outputs,
//   3. joins.
// Every kernel reads the counts from device memory, so the graph captured
// once is replayed for any request mix within the capacities. ps_batch_tune
// times candidate SM splits and trajectory tile widths on the current
// requests and keeps the fastest.
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>

#include "ps_costlane.cuh"
#include "ps_edgekern.cuh"

namespace ps {
namespace {

struct EdgeReq {           // one edge request as the device reads it
    const float* from;     // [n][D]
    const float* to;       // [n][D]
    const int* samples;    // [n] or NULL: the params rule
    uint8_t* valid;        // [n]
    float* cost;           // [n]
    int n, offset;         // rows, first packed row
};

struct TrajReq {
    const float* q;        // trajectory [T][D]; rollouts [rows][D][T]
    float* wp_cost;        // trajectory: [T] or NULL; rollouts: [rows*T] or [rows*D*T] (broadcast)
    float* traj_cost;      // [1] or NULL (trajectories only)
    float* grad;           // [T][D] or NULL (trajectories only)
    int T, offset;         // waypoints per row, first packed waypoint
    int rows;              // 1 for a trajectory, the rollout count otherwise
    int rollouts;          // 1: STOMP rollouts (reference layout, no gradient)
    int broadcast_d;       // rollouts: repeat each state cost over d
    int pad;
};

struct Counts {
    int n_edge_req, n_traj_req, n_edges, n_wp, n_roll;
};

constexpr int kFinishThreads = 128;   // same block width as ps_traj_cost's smoothness pass

// Packs every edge request's rows and resolves each edge's sample count.
__global__ void batch_gather_edges(const EdgeReq* __restrict__ req, const Counts* __restrict__ cnt,
                                   ps_edge_params P, int D, float* __restrict__ from, float* __restrict__ to,
                                   int* __restrict__ G) {
    const int nreq = cnt->n_edge_req;
    for (int r = blockIdx.x; r < nreq; r += gridDim.x) {
        const EdgeReq q = req[r];
        const size_t base = (size_t)q.offset * D;
        for (int i = threadIdx.x; i < q.n * D; i += blockDim.x) {
            from[base + i] = q.from[i];
            to[base + i] = q.to[i];
        }
        for (int i = threadIdx.x; i < q.n; i += blockDim.x) {
            const float* a = q.from + (size_t)i * D;
            const float* b = q.to + (size_t)i * D;
            G[q.offset + i] = edge_samples(P, q.samples, i, a, b, D, edge_length(a, b, D));
        }
    }
}

__global__ void batch_scatter_edges(const EdgeReq* __restrict__ req, const Counts* __restrict__ cnt,
                                    const uint8_t* __restrict__ valid, const float* __restrict__ cost) {
    const int nreq = cnt->n_edge_req;
    for (int r = blockIdx.x; r < nreq; r += gridDim.x) {
        const EdgeReq q = req[r];
        for (int i = threadIdx.x; i < q.n; i += blockDim.x) {
            q.valid[i] = valid[q.offset + i];
            q.cost[i] = cost[q.offset + i];
        }
    }
}

// Packs every trajectory's waypoints (waypoint-major); rollouts go from the
// reference layout [rows][D][T] to waypoint-major rows.
__global__ void batch_gather_traj(const TrajReq* __restrict__ req, const Counts* __restrict__ cnt, int D,
                                  float* __restrict__ q) {
    const int nreq = cnt->n_traj_req;
    for (int r = blockIdx.x; r < nreq; r += gridDim.x) {
        const TrajReq t = req[r];
        const size_t base = (size_t)t.offset * D;
        if (!t.rollouts) {
            for (int i = threadIdx.x; i < t.T * D; i += blockDim.x) q[base + i] = t.q[i];
        } else {
            const long long n = (long long)t.rows * t.T * D;
            for (long long i = threadIdx.x; i < n; i += blockDim.x) {   // i over the packed rows
                const int d = (int)(i % D);
                const long long w = i / D;
                const int row = (int)(w / t.T), tt = (int)(w - (long long)row * t.T);
                q[base + i] = t.q[((size_t)row * D + d) * t.T + tt];
            }
        }
    }
}

size_t waypoint_smem_bytes(const ps_model* m, const ps_scene_view* sv, int warps) {
    return lane_block_bytes(m, sv, warps, true);
}

// Cost and adjoint of every packed trajectory waypoint, and the cost alone of
// every packed rollout waypoint, kCostSub lanes per waypoint (kCostSlots
// consecutive packed waypoints per warp, ps_costlane.cuh). Trajectory
// waypoints fill [0, n_wp) of the packed rows, rollout waypoints
// [cap - n_roll, cap); a warp takes its waypoints from one range, so rollout
// warps run without the adjoint.
template <int kWarps>
__global__ void __launch_bounds__(kWarps * 32, 16 / kWarps) batch_waypoint_kernel(ModelDev md, ps_scene_view sv,
                                                                                 ps_cost_params P,
                                                                                 const Counts* __restrict__ cnt,
                                                                                 const float* __restrict__ q,
                                                                                 float* __restrict__ wp_cost,
                                                                                 float* __restrict__ grad, int cap) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    const int n_wp = cnt->n_wp, n_roll = cnt->n_roll;
    const int chunks_a = (n_wp + kCostSlots - 1) / kCostSlots, chunks = chunks_a + (n_roll + kCostSlots - 1) / kCostSlots;
    if (blockIdx.x * kWarps >= chunks) return;   // nothing for this block: skip staging
    if (!stage_model(md, smem, &mbar)) {   // fail closed: NaN costs and gradient rows
        const float nan = __int_as_float(0x7fc00000);
        cost_fail_closed(md, n_wp, kWarps * kCostSlots, [&](long long k, int D) {
            wp_cost[k] = nan;
            for (int d = 0; d < D; ++d) grad[(size_t)k * D + d] = nan;
        });
        cost_fail_closed(md, n_roll, kWarps * kCostSlots, [&](long long k, int D) { wp_cost[cap - n_roll + k] = nan; });
        return;
    }
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof, NJ = M.H->n_joints;
    ObbPrep* obbs = reinterpret_cast<ObbPrep*>(smem + md.bytes_core);
    const int nob = max(sv.n_obbs, 1);
    int* orig = reinterpret_cast<int*>(obbs + nob);
    LayerPrep* layers = reinterpret_cast<LayerPrep*>(orig + ((nob + 3) & ~3));
    SceneSmem sc;
    stage_scene(sv, obbs, orig, layers, counters, &bmax, sc);
    const CostBlock cb = cost_block_setup(reinterpret_cast<unsigned char*>(layers + PS_MAX_LAYERS), M, sc, sv.n_obbs);
    __syncthreads();
    box_limits(sc, const_cast<float4*>(cb.obs));
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / kCostSub, u = lane % kCostSub;
    const int NS = M.H->n_spheres;
    const LaneScratch ws = lane_carve(
        reinterpret_cast<unsigned char*>(cb.wbase) + (size_t)warp * lane_warp_bytes(NJ, NS, D, sv.n_obbs, true), NJ,
        NS, D, true);
    LaneStats st;
    for (int c = blockIdx.x * kWarps + warp; c < chunks; c += gridDim.x * kWarps) {
        const bool traj = c < chunks_a;   // uniform over the warp
        const int lo = traj ? 0 : cap - n_roll, hi = traj ? n_wp : cap;
        const int k = lo + (traj ? c : c - chunks_a) * kCostSlots + slot;
        const int kc = k < hi ? k : hi - 1;   // past the end: repeat the last waypoint
        for (int d = u; d < D; d += kCostSub) lane_put_q(ws, slot, d, q[(size_t)kc * D + d]);
        __syncwarp();
        st.zero();
        if (traj) {
            const float v = lane_cost<true, false>(M, md, sc, sv, P, cb, ws, st);
            if (k < hi) {
                if (u == 0) wp_cost[k] = v;
                lane_write_grad(M, cb, ws, grad + (size_t)k * D, 1);
            }
        } else {
            const float v = lane_cost<false, false>(M, md, sc, sv, P, cb, ws, st);
            if (k < hi && u == 0) wp_cost[k] = v;
        }
    }
}

// Per-warp scratch of the work-queue kernel. Every warp holds an edge chunk's
// (32 configurations and the broad phase's candidate list); the first
// cost_warps warps of a block also take waypoint groups and hold the
// lane-group scratch in the same region, one item at a time. Fewer such
// warps leave room for more resident blocks, so more warps for edge items.
__host__ __device__ inline size_t work_edge_bytes(int D, int n_obbs) {
    return ((size_t)32 * D * 4 + (size_t)((n_obbs > 1 ? n_obbs : 1) + 7) / 8 * 8 * 2 + 15) & ~size_t(15);
}
__host__ __device__ inline size_t work_cost_bytes(int NJ, int NS, int D, int n_obbs) {
    const size_t edge = work_edge_bytes(D, n_obbs);
    const size_t cost = lane_warp_bytes(NJ, NS, D, n_obbs, true);
    return ((edge > cost ? edge : cost) + 15) & ~size_t(15);
}
__host__ __device__ inline size_t work_warp_offset(int warp, int cost_warps, int NJ, int NS, int D, int n_obbs) {
    const size_t cb = work_cost_bytes(NJ, NS, D, n_obbs), eb = work_edge_bytes(D, n_obbs);
    return warp < cost_warps ? (size_t)warp * cb : (size_t)cost_warps * cb + (size_t)(warp - cost_warps) * eb;
}

size_t work_smem_bytes(const ps_model* m, const ps_scene_view* sv, int warps, int cost_warps) {
    const size_t tables = lane_block_bytes(m, sv, 0, true);
    return tables + work_warp_offset(warps, cost_warps, m->info.n_joints, m->info.n_spheres, m->info.n_dof,
                                     sv->n_obbs);
}

// The whole batch as one persistent work queue. Every warp pulls, from
// global counters, first the persistent edge path's chunk-major items of
// this pass (hdr->head[pass]: a chunk of 32 consecutive samples of one edge,
// skipped once the edge is retired), then, in the last pass, waypoint groups
// (hdr->wp_next: kCostSlots consecutive packed waypoints; trajectory groups
// with the adjoint, rollout groups without it), until both are drained.
// Pass 0 holds only chunk round 0 when the edges are too few to keep round 0
// ahead of the later rounds (the persistent edge path's split rule); pass 1
// then holds the later rounds and the waypoint groups. The edge
// items are processed exactly as by edges_queue_kernel and the waypoint
// groups exactly as by batch_waypoint_kernel, so every output has the same
// bits as with the two kernels side by side.
template <int kMode, int kW>
__global__ void __launch_bounds__(kW * 32, 16 / kW)
    batch_work_kernel(ModelDev md, ps_scene_view sv, ps_edge_params EP, ps_cost_params CP,
                      const Counts* __restrict__ cnt, const float* __restrict__ from, const float* __restrict__ to,
                      EdgeWs* hdr, const int* __restrict__ Gs, int* bad, int* clr, int* done,
                      const float* __restrict__ q, float* __restrict__ wp_cost, float* __restrict__ grad, int cap,
                      int pass, int cost_warps) {
    const int n_edges = cnt->n_edges, n_wp = cnt->n_wp, n_roll = cnt->n_roll;
    const int max_rounds = *((volatile int*)&hdr->max_rounds);
    const bool split = (long long)n_edges < 8ll * gridDim.x * kW;
    // the waypoint groups follow the edge items of the last pass, where they
    // fill the tail of the edge work
    const int chunks_a = (n_wp + kCostSlots - 1) / kCostSlots;
    const int chunks = pass == (split ? 1 : 0) ? chunks_a + (n_roll + kCostSlots - 1) / kCostSlots : 0;
    const int r_lo = pass == 0 ? 0 : (split ? 1 : max_rounds);
    const int r_hi = pass == 0 ? (split ? min(max_rounds, 1) : max_rounds) : max_rounds;
    const long long total = (long long)max(r_hi - r_lo, 0) * n_edges;   // edge items of this pass
    if (total == 0 && chunks == 0) return;   // uniform over the grid: nothing staged yet
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ int counters[4];
    __shared__ float bmax;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / kCostSub, u = lane % kCostSub;
    if (!stage_model(md, smem, &mbar)) {
        // fail closed: the edges come back invalid (finalize, timed_out) and
        // the waypoint groups this block pulls NaN
        if (threadIdx.x == 0 && total > 0) atomicExch(&hdr->timed_out, 1);
        const int D = reinterpret_cast<const BlobHeader*>(md.blob)->n_dof;
        const float nan = __int_as_float(0x7fc00000);
        while (chunks > 0 && warp < cost_warps) {   // (a pass without groups leaves the counter alone)
            int c = 0;
            if (lane == 0) c = atomicAdd(&hdr->wp_next, 1);
            c = __shfl_sync(kFull, c, 0);
            if (c >= chunks) break;
            const bool traj = c < chunks_a;
            const int lo = traj ? 0 : cap - n_roll, hi = traj ? n_wp : cap;
            const int k = lo + (traj ? c : c - chunks_a) * kCostSlots + slot;
            if (k < hi) {
                if (u == 0) wp_cost[k] = nan;
                if (traj)
                    for (int d = u; d < D; d += kCostSub) grad[(size_t)k * D + d] = nan;
            }
        }
        return;
    }
    const ModelSmem M = model_view(smem);
    const int D = M.H->n_dof, NJ = M.H->n_joints, NS = M.H->n_spheres;
    ObbPrep* obbs = reinterpret_cast<ObbPrep*>(smem + md.bytes_core);
    const int nob = max(sv.n_obbs, 1);
    int* orig = reinterpret_cast<int*>(obbs + nob);
    LayerPrep* layers = reinterpret_cast<LayerPrep*>(orig + ((nob + 3) & ~3));
    SceneSmem sc;
    stage_scene(sv, obbs, orig, layers, counters, &bmax, sc);
    const CostBlock cb = cost_block_setup(reinterpret_cast<unsigned char*>(layers + PS_MAX_LAYERS), M, sc, sv.n_obbs);
    __syncthreads();
    box_limits(sc, const_cast<float4*>(cb.obs));
    __syncthreads();
    unsigned char* wbase =
        reinterpret_cast<unsigned char*>(cb.wbase) + work_warp_offset(warp, cost_warps, NJ, NS, D, sv.n_obbs);
    LaneStats st;
    st.zero();

    // ---- edge chunk items (edges_queue_kernel's loop) ----
    if (total > 0) {
        float* eq = reinterpret_cast<float*>(wbase);
        WarpScratch ws{eq, reinterpret_cast<uint16_t*>(eq + 32 * D), cb.obs};
        unsigned long long* head = &hdr->head[pass == 0 ? 0 : 1];
        const unsigned long long deadline = *((volatile unsigned long long*)&hdr->deadline);
        const int grab = EP.grab > 0 ? min(EP.grab, 32) : (int)max(1ll, min(32ll, total / ((long long)gridDim.x * kW * 2)));
        volatile int* vbad = bad;
        for (;;) {
            unsigned long long base = 0;
            if (lane == 0) {
                if (deadline && global_ns() > deadline) {
                    atomicExch(&hdr->timed_out, 1);
                    base = (unsigned long long)total;
                } else {
                    base = atomicAdd(head, (unsigned long long)grab);
                }
            }
            base = __shfl_sync(kFull, base, 0);
            if ((long long)base >= total) break;
            const long long item = (long long)base + lane;
            int e = -1, k = 0, G = 0;
            bool live = false;
            if (lane < grab && item < total) {
                if (total < (1ll << 31)) {   // 32-bit division in the common case
                    k = (int)((unsigned)item / (unsigned)n_edges);
                    e = (int)((unsigned)item - (unsigned)k * (unsigned)n_edges);
                } else {
                    k = (int)(item / n_edges);
                    e = (int)(item - (long long)k * n_edges);
                }
                k += r_lo;
                G = __ldg(Gs + e);
                const ChunkOrder ord(G);
                if (k < ord.rounds()) {
                    k = ord.chunk(k);
                    live = k < ord.nc && (EP.compute_clearance || vbad[e] == 0);
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
                if (!EP.compute_clearance && retired) continue;
                float cm = FLT_MAX;
                const bool h = kMode ? process_chunk_fast<false, kMode == 2>(M, sc, sv, EP, from, to, ee, GG, kk, ws, st)
                                     : process_chunk(M, sc, sv, EP, from, to, ee, GG, kk, ws,
                                                     EP.compute_clearance ? &cm : nullptr, st);
                if (lane == 0) {
                    if (h) vbad[ee] = 1;
                    if (EP.compute_clearance) atomicMin(clr + ee, ordered_float(cm));
                    if (deadline) atomicAdd(done + ee, 1);
                }
            }
        }
    }

    // ---- waypoint groups (batch_waypoint_kernel's loop) ----
    if (chunks > 0 && warp < cost_warps) {
        const LaneScratch ws = lane_carve(wbase, NJ, NS, D, true);
        for (;;) {
            int c = 0;
            if (lane == 0) c = atomicAdd(&hdr->wp_next, 1);
            c = __shfl_sync(kFull, c, 0);
            if (c >= chunks) break;
            const bool traj = c < chunks_a;   // uniform over the warp
            const int lo = traj ? 0 : cap - n_roll, hi = traj ? n_wp : cap;
            const int k = lo + (traj ? c : c - chunks_a) * kCostSlots + slot;
            const int kc = k < hi ? k : hi - 1;   // past the end: repeat the last waypoint
            __syncwarp();   // the previous group's readers of the scratch are done
            for (int d = u; d < D; d += kCostSub) lane_put_q(ws, slot, d, q[(size_t)kc * D + d]);
            __syncwarp();
            if (traj) {
                const float v = lane_cost<true, false>(M, md, sc, sv, CP, cb, ws, st);
                if (k < hi) {
                    if (u == 0) wp_cost[k] = v;
                    lane_write_grad(M, cb, ws, grad + (size_t)k * D, 1);
                }
            } else {
                const float v = lane_cost<false, false>(M, md, sc, sv, CP, cb, ws, st);
                if (k < hi && u == 0) wp_cost[k] = v;
            }
        }
    }
}

// One block per trajectory request: outputs waypoint costs, the gradient
// (adjoint + smoothness) and the total, exactly as ps_traj_cost computes them.
__global__ void __launch_bounds__(kFinishThreads) batch_traj_finish(const TrajReq* __restrict__ req,
                                                                    const Counts* __restrict__ cnt, int D,
                                                                    ps_cost_params P, const float* __restrict__ q,
                                                                    const float* __restrict__ wp_cost,
                                                                    const float* __restrict__ grad) {
    extern __shared__ float sh[];
    const int nreq = cnt->n_traj_req;
    for (int r = blockIdx.x; r < nreq; r += gridDim.x) {
        const TrajReq t = req[r];
        const float* qr = q + (size_t)t.offset * D;
        const float* wr = wp_cost + t.offset;
        if (t.rollouts) {   // state costs only, in the reference layout
            const long long n = (long long)t.rows * t.T;
            for (long long i = threadIdx.x; i < n; i += blockDim.x) {
                if (t.broadcast_d) {
                    const long long row = i / t.T, tt = i - row * t.T;
                    for (int d = 0; d < D; ++d) t.wp_cost[((size_t)row * D + d) * t.T + tt] = wr[i];
                } else {
                    t.wp_cost[i] = wr[i];
                }
            }
            continue;   // uniform over the block
        }
        if (t.wp_cost)
            for (int i = threadIdx.x; i < t.T; i += blockDim.x) t.wp_cost[i] = wr[i];
        if (t.grad)
            for (int i = threadIdx.x; i < t.T * D; i += blockDim.x) t.grad[i] = grad[(size_t)t.offset * D + i];
        __syncthreads();   // the copied rows are read back by other threads below
        if (!t.traj_cost && !(t.grad && P.smoothness_weight != 0.0f)) continue;
        float* g = t.grad;
        const float tot = traj_smooth_block([&](int tt, int d) { return qr[(size_t)tt * D + d]; },
                                            [&](int tt, int d, float v) { g[(size_t)tt * D + d] += v; },
                                            [&](int tt) { return wr[tt]; }, t.T, D, P, g != nullptr, sh);
        if (threadIdx.x == 0 && t.traj_cost) *t.traj_cost = tot;
    }
}

size_t align256b(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace ps

using namespace ps;

struct ps_batch {
    const ps_model* model = nullptr;
    ps_batch_limits lim{};
    std::vector<EdgeReq> ereq;
    std::vector<TrajReq> treq;
    int n_edges = 0, n_wp = 0, n_roll = 0;   // trajectory waypoints from 0 up, rollout waypoints from the top
    // pinned mirrors read by every replay
    EdgeReq* h_ereq = nullptr;
    TrajReq* h_treq = nullptr;
    Counts* h_cnt = nullptr;
    // one device allocation holds every packed buffer
    void* dmem = nullptr;
    EdgeReq* d_ereq = nullptr;
    TrajReq* d_treq = nullptr;
    Counts* d_cnt = nullptr;
    float *d_from = nullptr, *d_to = nullptr, *d_len = nullptr, *d_cost = nullptr;
    int *d_given = nullptr, *d_G = nullptr, *d_bad = nullptr, *d_clr = nullptr, *d_done = nullptr;
    uint8_t* d_valid = nullptr;
    EdgeWs* d_hdr = nullptr;
    float *d_q = nullptr, *d_wp_cost = nullptr, *d_grad = nullptr;
    // captured graph and the configuration it was captured for
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
    cudaStream_t cap0 = nullptr, cap1 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, done = nullptr;
    bool launched = false;
    // tuning state
    float edge_share = 1.0f;   // of the edge kernel's full-occupancy grid
    float traj_share = 0.5f;   // of the trajectory kernel's full-occupancy grid
    int traj_threads = 256;   // threads per block of the trajectory kernel (kCostSub per waypoint)
    int traj_tile = 1;        // kept for the tuning record: always 1
    int layout = 0;           // 0: edge queue and waypoint kernel side by side; 1: one work-queue kernel
    int work_threads = 256;   // threads per block of the work-queue kernel
    int work_cost_warps = 8;  // warps per block of it that also take waypoint groups
};

namespace {

struct LaunchPlan {
    int mode = 0;
    void (*qk)(ModelDev, ps_scene_view, ps_edge_params, const float*, const float*, int, EdgeWs*, const int*, int*,
               int*, int*, unsigned long long*, int, const int*, const int*) = nullptr;
    void (*wk)(ModelDev, ps_scene_view, ps_cost_params, const Counts*, const float*, float*, float*, int) = nullptr;
    void (*work)(ModelDev, ps_scene_view, ps_edge_params, ps_cost_params, const Counts*, const float*, const float*,
                 EdgeWs*, const int*, int*, int*, int*, const float*, float*, float*, int, int, int) = nullptr;
    size_t qsmem = 0, wsmem = 0, fsmem = 0, ssmem = 0, ksmem = 0;
    int qgrid = 1, wgrid = 1, req_grid_e = 1, req_grid_t = 1, pgrid = 1, sgrid = 1, kgrid = 1;
    ProbePlan probe;
};

using WorkKernel = decltype(LaunchPlan::work);

WorkKernel pick_work_kernel(int mode, int threads) {
    if (threads == 128)
        return mode == 1 ? batch_work_kernel<1, 4> : (mode == 2 ? batch_work_kernel<2, 4> : batch_work_kernel<0, 4>);
    return mode == 1 ? batch_work_kernel<1, 8> : (mode == 2 ? batch_work_kernel<2, 8> : batch_work_kernel<0, 8>);
}

using WaypointKernel = void (*)(ModelDev, ps_scene_view, ps_cost_params, const Counts*, const float*, float*, float*,
                                int);

WaypointKernel pick_waypoint_kernel(int threads) {
    return threads == 128 ? batch_waypoint_kernel<4> : batch_waypoint_kernel<8>;
}

// Everything that is not a stream operation happens before the capture.
int plan_launch(ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep, LaunchPlan& L) {
    const ps_model* m = b->model;
    const int sms = sm_count();
    if (b->lim.max_edges > 0) {
        L.mode = fast_path(m, sv, ep);
        L.qk = pick(L.mode, false, edges_queue_kernel<0, false>, edges_queue_kernel<0, true>,
                    edges_queue_kernel<1, false>, edges_queue_kernel<1, true>, edges_queue_kernel<2, false>,
                    edges_queue_kernel<2, true>);
        L.qsmem = edge_smem_bytes(m, sv);
        PS_TRY_CUDA(allow_smem((const void*)L.qk, L.qsmem));
        int per_sm = 0;
        PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.qk, kEdgeThreads, L.qsmem));
        if (per_sm < 1) return set_error(PS_EINVAL, "edge kernel does not fit on an SM with this scene");
        L.qgrid = std::max(1, (int)(b->edge_share * sms * per_sm + 0.5f));
        if (int rc = plan_probe(m, sv, L.mode, false, b->edge_share, b->lim.max_edges, ep->probe, L.probe)) return rc;
        L.pgrid = std::max(1, std::min((b->lim.max_edges + 255) / 256, sms * 4));
        L.req_grid_e = std::max(1, std::min(b->lim.max_edge_requests, sms * 8));
        if (ep->check_self) {
            if (int rc = check_self_fits(m)) return rc;
            L.ssmem = self_lane_smem_bytes(m);
            PS_TRY_CUDA(allow_smem((const void*)edges_self_kernel, L.ssmem));
            int s_per_sm = 0;
            PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s_per_sm, edges_self_kernel, kSelfThreads,
                                                                      L.ssmem));
            if (s_per_sm < 1) return set_error(PS_EINVAL, "self-check kernel does not fit on an SM with this model");
            L.sgrid = std::max(1, std::min(b->lim.max_edges, (int)(b->edge_share * sms * s_per_sm + 0.5f)));
        }
    }
    if (b->lim.max_waypoints > 0) {
        const int tt = b->traj_threads;
        L.wsmem = waypoint_smem_bytes(m, sv, tt / 32);
        L.wk = pick_waypoint_kernel(tt);
        int per_sm = 0;
        PS_TRY_CUDA(allow_smem((const void*)L.wk, L.wsmem));
        PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.wk, tt, L.wsmem));
        if (per_sm < 1) return set_error(PS_EINVAL, "trajectory kernel does not fit on an SM with this model/scene");
        const int per_block = tt / kCostSub;   // waypoints per block
        const int cap_blocks = (b->lim.max_waypoints + per_block - 1) / per_block;
        L.wgrid = std::max(1, std::min(cap_blocks, (int)(b->traj_share * sms * per_sm + 0.5f)));
        L.fsmem = (size_t)(2 * (b->lim.max_traj_len + 12) + kFinishThreads) * sizeof(float);
        if (L.fsmem > 48 * 1024)
            PS_TRY_CUDA(allow_smem((const void*)batch_traj_finish, L.fsmem));
        L.req_grid_t = std::max(1, std::min(b->lim.max_traj_requests, sms * 8));
    }
    if (b->layout == 1) {   // one work-queue kernel for edge chunks and waypoint groups
        const int mode = b->lim.max_edges > 0 ? L.mode : 1;
        const int kt = b->work_threads;
        L.work = pick_work_kernel(mode, kt);
        L.ksmem = work_smem_bytes(m, sv, kt / 32, std::min(b->work_cost_warps, kt / 32));
        PS_TRY_CUDA(allow_smem((const void*)L.work, L.ksmem));
        int per_sm = 0;
        PS_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.work, kt, L.ksmem));
        if (per_sm < 1) return set_error(PS_EINVAL, "work-queue kernel does not fit on an SM with this model/scene");
        L.kgrid = std::max(1, sms * per_sm);
    }
    return PS_OK;
}

// Layout 1: one stream; gathers, edge prep and the end-sample probe, then
// the work-queue kernel twice (split: round 0, then the later rounds and the
// waypoint groups; otherwise every round and the waypoint groups, then
// nothing), the self pass, finalize, scatter and the trajectory outputs.
void record_work_graph(ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep, const ps_cost_params* cp,
                       const LaunchPlan& L) {
    const ps_model* m = b->model;
    const int D = m->info.n_dof;
    cudaStream_t s0 = b->cap0;
    const int* n_dev = &b->d_cnt->n_edges;
    const bool edges = b->lim.max_edges > 0, trajs = b->lim.max_waypoints > 0;
    cudaMemsetAsync(b->d_hdr, 0, sizeof(EdgeWs), s0);
    if (edges) {
        batch_gather_edges<<<L.req_grid_e, 128, 0, s0>>>(b->d_ereq, b->d_cnt, *ep, D, b->d_from, b->d_to, b->d_given);
        edges_prep_kernel<<<L.pgrid, 256, 0, s0>>>(*ep, b->d_from, b->d_to, b->d_given, b->lim.max_edges, D, b->d_hdr,
                                                   b->d_G, b->d_len, b->d_bad, b->d_clr, b->d_done, n_dev);
        if (L.probe.k)
            L.probe.k<<<L.probe.grid, kProbeThreads, L.probe.smem, s0>>>(m->dev, *sv, *ep, b->d_from, b->d_to,
                                                                          b->lim.max_edges, b->d_hdr, b->d_G,
                                                                          b->d_bad, nullptr, n_dev, PrepArgs{});
    }
    if (trajs) batch_gather_traj<<<L.req_grid_t, 128, 0, s0>>>(b->d_treq, b->d_cnt, D, b->d_q);
    for (int pass = 0; pass < 2; ++pass)
        L.work<<<L.kgrid, b->work_threads, L.ksmem, s0>>>(m->dev, *sv, *ep, *cp, b->d_cnt, b->d_from, b->d_to,
                                                          b->d_hdr, b->d_G, b->d_bad, b->d_clr, b->d_done, b->d_q,
                                                          b->d_wp_cost, b->d_grad, b->lim.max_waypoints, pass,
                                                          std::min(b->work_cost_warps, b->work_threads / 32));
    if (edges) {
        if (ep->check_self)
            edges_self_kernel<<<L.sgrid, kSelfThreads, L.ssmem, s0>>>(m->dev, *ep, b->d_from, b->d_to, b->d_given,
                                                                      b->lim.max_edges, b->d_G, b->d_bad, nullptr,
                                                                      nullptr, b->d_hdr, nullptr, n_dev);
        edges_finalize_kernel<<<L.pgrid, 256, 0, s0>>>(b->lim.max_edges, *ep, b->d_bad, b->d_len, b->d_clr, b->d_done,
                                                       b->d_G, b->d_hdr, b->d_valid, b->d_cost, nullptr, n_dev);
        batch_scatter_edges<<<L.req_grid_e, 128, 0, s0>>>(b->d_ereq, b->d_cnt, b->d_valid, b->d_cost);
    }
    if (trajs)
        batch_traj_finish<<<L.req_grid_t, kFinishThreads, L.fsmem, s0>>>(b->d_treq, b->d_cnt, D, *cp, b->d_q,
                                                                         b->d_wp_cost, b->d_grad);
}

void record_graph(ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep, const ps_cost_params* cp,
                  const LaunchPlan& L) {
    const ps_model* m = b->model;
    const int D = m->info.n_dof;
    cudaStream_t s0 = b->cap0, s1 = b->cap1;
    cudaMemcpyAsync(b->d_ereq, b->h_ereq, sizeof(EdgeReq) * std::max(b->lim.max_edge_requests, 1),
                    cudaMemcpyHostToDevice, s0);
    cudaMemcpyAsync(b->d_treq, b->h_treq, sizeof(TrajReq) * std::max(b->lim.max_traj_requests, 1),
                    cudaMemcpyHostToDevice, s0);
    cudaMemcpyAsync(b->d_cnt, b->h_cnt, sizeof(Counts), cudaMemcpyHostToDevice, s0);
    if (b->layout == 1) {
        record_work_graph(b, sv, ep, cp, L);
        return;
    }
    cudaEventRecord(b->fork, s0);
    cudaStreamWaitEvent(s1, b->fork, 0);
    if (b->lim.max_edges > 0) {   // edge branch on s0
        const int* n_dev = &b->d_cnt->n_edges;
        cudaMemsetAsync(b->d_hdr, 0, sizeof(EdgeWs), s0);
        batch_gather_edges<<<L.req_grid_e, 128, 0, s0>>>(b->d_ereq, b->d_cnt, *ep, D, b->d_from, b->d_to, b->d_given);
        edges_prep_kernel<<<L.pgrid, 256, 0, s0>>>(*ep, b->d_from, b->d_to, b->d_given, b->lim.max_edges, D, b->d_hdr,
                                                   b->d_G, b->d_len, b->d_bad, b->d_clr, b->d_done, n_dev);
        if (L.probe.k)
            L.probe.k<<<L.probe.grid, kProbeThreads, L.probe.smem, s0>>>(m->dev, *sv, *ep, b->d_from, b->d_to,
                                                                          b->lim.max_edges, b->d_hdr, b->d_G,
                                                                          b->d_bad, nullptr, n_dev, PrepArgs{});
        L.qk<<<L.qgrid, kEdgeThreads, L.qsmem, s0>>>(m->dev, *sv, *ep, b->d_from, b->d_to, b->lim.max_edges, b->d_hdr,
                                                    b->d_G, b->d_bad, b->d_clr, b->d_done, nullptr, 0, n_dev, nullptr);
        L.qk<<<L.qgrid, kEdgeThreads, L.qsmem, s0>>>(m->dev, *sv, *ep, b->d_from, b->d_to, b->lim.max_edges, b->d_hdr,
                                                    b->d_G, b->d_bad, b->d_clr, b->d_done, nullptr, 1, n_dev, nullptr);
        if (ep->check_self)
            edges_self_kernel<<<L.sgrid, kSelfThreads, L.ssmem, s0>>>(m->dev, *ep, b->d_from, b->d_to, b->d_given,
                                                                      b->lim.max_edges, b->d_G, b->d_bad, nullptr,
                                                                      nullptr, b->d_hdr, nullptr, n_dev);
        edges_finalize_kernel<<<L.pgrid, 256, 0, s0>>>(b->lim.max_edges, *ep, b->d_bad, b->d_len, b->d_clr, b->d_done,
                                                       b->d_G, b->d_hdr, b->d_valid, b->d_cost, nullptr, n_dev);
        batch_scatter_edges<<<L.req_grid_e, 128, 0, s0>>>(b->d_ereq, b->d_cnt, b->d_valid, b->d_cost);
    }
    if (b->lim.max_waypoints > 0) {   // trajectory branch on s1
        batch_gather_traj<<<L.req_grid_t, 128, 0, s1>>>(b->d_treq, b->d_cnt, D, b->d_q);
        L.wk<<<L.wgrid, b->traj_threads, L.wsmem, s1>>>(m->dev, *sv, *cp, b->d_cnt, b->d_q, b->d_wp_cost, b->d_grad,
                                                        b->lim.max_waypoints);
        batch_traj_finish<<<L.req_grid_t, kFinishThreads, L.fsmem, s1>>>(b->d_treq, b->d_cnt, D, *cp, b->d_q,
                                                                         b->d_wp_cost, b->d_grad);
    }
    cudaEventRecord(b->join, s1);
    cudaStreamWaitEvent(s0, b->join, 0);
}

int batch_capture(ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep, const ps_cost_params* cp) {
    LaunchPlan L;
    if (int rc = plan_launch(b, sv, ep, L)) return rc;
    PS_TRY_CUDA(cudaStreamBeginCapture(b->cap0, cudaStreamCaptureModeThreadLocal));
    record_graph(b, sv, ep, cp, L);
    cudaGraph_t g = nullptr;
    const cudaError_t le = cudaGetLastError();
    cudaError_t e = cudaStreamEndCapture(b->cap0, &g);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_error(le != cudaSuccess ? le : e, "capture of the batch graph");
    }
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_error(e, "instantiate the batch graph");
    return PS_OK;
}

std::vector<unsigned char> make_key(const ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep,
                                    const ps_cost_params* cp) {
    std::vector<unsigned char> k(sizeof(*sv) + sizeof(*ep) + sizeof(*cp) + 2 * sizeof(float) + 6 * sizeof(int));
    unsigned char* p = k.data();
    auto put = [&](const void* src, size_t n) {
        std::memcpy(p, src, n);
        p += n;
    };
    put(sv, sizeof(*sv));
    put(ep, sizeof(*ep));
    put(cp, sizeof(*cp));
    put(&b->edge_share, sizeof(float));
    put(&b->traj_share, sizeof(float));
    put(&b->traj_threads, sizeof(int));
    put(&b->traj_tile, sizeof(int));
    put(&b->layout, sizeof(int));
    put(&b->work_threads, sizeof(int));
    put(&b->work_cost_warps, sizeof(int));
    put(&b->model->dev.stage_polls, sizeof(int));   // kernels get the model by value at capture
    return k;
}

void release(ps_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->cap0) cudaStreamDestroy(b->cap0);
    if (b->cap1) cudaStreamDestroy(b->cap1);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->done) cudaEventDestroy(b->done);
    if (b->h_ereq) cudaFreeHost(b->h_ereq);
    if (b->h_treq) cudaFreeHost(b->h_treq);
    if (b->h_cnt) cudaFreeHost(b->h_cnt);
    if (b->dmem) cudaFree(b->dmem);
    delete b;
}

}  // namespace

extern "C" int ps_batch_create(const ps_model* m, const ps_batch_limits* lim, ps_batch** out) {
    clear_error();
    if (!m || !lim || !out) return set_error(PS_EINVAL, "NULL argument");
    if (int rc = check_model_device(m)) return rc;
    *out = nullptr;
    if (lim->max_edge_requests < 0 || lim->max_edges < 0 || lim->max_traj_requests < 0 || lim->max_waypoints < 0 ||
        lim->max_traj_len < 0)
        return set_error(PS_EINVAL, "negative capacity");
    if (lim->max_edges > 0 && lim->max_edge_requests <= 0)
        return set_error(PS_EINVAL, "max_edge_requests must be > 0 when max_edges > 0");
    if (lim->max_waypoints > 0 && (lim->max_traj_requests <= 0 || lim->max_traj_len <= 0))
        return set_error(PS_EINVAL, "max_traj_requests and max_traj_len must be > 0 when max_waypoints > 0");
    if (lim->max_traj_len > PS_MAX_TRAJ_LEN) return set_error(PS_EINVAL, "max_traj_len exceeds PS_MAX_TRAJ_LEN");
    if (m->info.n_joints > 255) return set_error(PS_EINVAL, "too many joints");
    ps_batch* b = new ps_batch();
    b->model = m;
    b->lim = *lim;
    const int D = m->info.n_dof;
    const size_t E = (size_t)std::max(lim->max_edges, 1), W = (size_t)std::max(lim->max_waypoints, 1);
    const size_t RE = (size_t)std::max(lim->max_edge_requests, 1), RT = (size_t)std::max(lim->max_traj_requests, 1);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align256b(bytes);
        return o;
    };
    const size_t o_ereq = take(sizeof(EdgeReq) * RE), o_treq = take(sizeof(TrajReq) * RT), o_cnt = take(sizeof(Counts));
    const size_t o_from = take(4 * E * D), o_to = take(4 * E * D), o_len = take(4 * E), o_cost = take(4 * E);
    const size_t o_given = take(4 * E), o_G = take(4 * E), o_bad = take(4 * E), o_clr = take(4 * E),
                 o_done = take(4 * E);
    const size_t o_valid = take(E), o_hdr = take(sizeof(EdgeWs));
    const size_t o_q = take(4 * W * D), o_wpc = take(4 * W), o_grad = take(4 * W * D);
    cudaError_t e = cudaMalloc(&b->dmem, off);
    if (e != cudaSuccess) {
        b->dmem = nullptr;
        release(b);
        return set_error(PS_ENOMEM, std::string("batch buffers: ") + cudaGetErrorString(e));
    }
    unsigned char* base = (unsigned char*)b->dmem;
    b->d_ereq = (EdgeReq*)(base + o_ereq);
    b->d_treq = (TrajReq*)(base + o_treq);
    b->d_cnt = (Counts*)(base + o_cnt);
    b->d_from = (float*)(base + o_from);
    b->d_to = (float*)(base + o_to);
    b->d_len = (float*)(base + o_len);
    b->d_cost = (float*)(base + o_cost);
    b->d_given = (int*)(base + o_given);
    b->d_G = (int*)(base + o_G);
    b->d_bad = (int*)(base + o_bad);
    b->d_clr = (int*)(base + o_clr);
    b->d_done = (int*)(base + o_done);
    b->d_valid = base + o_valid;
    b->d_hdr = (EdgeWs*)(base + o_hdr);
    b->d_q = (float*)(base + o_q);
    b->d_wp_cost = (float*)(base + o_wpc);
    b->d_grad = (float*)(base + o_grad);
    if (cudaHostAlloc((void**)&b->h_ereq, sizeof(EdgeReq) * RE, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&b->h_treq, sizeof(TrajReq) * RT, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void**)&b->h_cnt, sizeof(Counts), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        release(b);
        return set_error(PS_ENOMEM, "pinned request tables");
    }
    std::memset(b->h_ereq, 0, sizeof(EdgeReq) * RE);
    std::memset(b->h_treq, 0, sizeof(TrajReq) * RT);
    std::memset(b->h_cnt, 0, sizeof(Counts));
    if (cudaStreamCreateWithFlags(&b->cap0, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->cap1, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
        const cudaError_t le = cudaGetLastError();
        release(b);
        return cuda_error(le, "batch streams/events");
    }
    *out = b;
    return PS_OK;
}

extern "C" int ps_batch_destroy(ps_batch* b) {
    clear_error();
    if (!b) return PS_OK;
    if (b->launched) cudaEventSynchronize(b->done);
    release(b);
    return PS_OK;
}

extern "C" int ps_batch_clear(ps_batch* b) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "NULL batch");
    b->ereq.clear();
    b->treq.clear();
    b->n_edges = b->n_wp = b->n_roll = 0;
    return PS_OK;
}

extern "C" int ps_batch_add_edges(ps_batch* b, const float* from, const float* to, const int* samples, int n,
                                  uint8_t* valid, float* cost) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "NULL batch");
    if (n < 0) return set_error(PS_EINVAL, "negative edge count");
    if (n > 0 && (!from || !to || !valid || !cost)) return set_error(PS_EINVAL, "NULL edge buffer");
    if ((int)b->ereq.size() >= b->lim.max_edge_requests) return set_error(PS_EINVAL, "too many edge requests");
    if ((long long)b->n_edges + n > b->lim.max_edges) return set_error(PS_EINVAL, "edge capacity exceeded");
    b->ereq.push_back(EdgeReq{from, to, samples, valid, cost, n, b->n_edges});
    b->n_edges += n;
    return PS_OK;
}

extern "C" int ps_batch_add_trajectory(ps_batch* b, const float* q, int T, float* waypoint_cost, float* traj_cost,
                                       float* grad) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "NULL batch");
    if (T <= 0 || !q) return set_error(PS_EINVAL, "empty trajectory or NULL q");
    if (T > b->lim.max_traj_len) return set_error(PS_EINVAL, "trajectory longer than max_traj_len");
    if ((int)b->treq.size() >= b->lim.max_traj_requests) return set_error(PS_EINVAL, "too many trajectory requests");
    if ((long long)b->n_wp + b->n_roll + T > b->lim.max_waypoints)
        return set_error(PS_EINVAL, "waypoint capacity exceeded");
    b->treq.push_back(TrajReq{q, waypoint_cost, traj_cost, grad, T, b->n_wp, 1, 0, 0, 0});
    b->n_wp += T;
    return PS_OK;
}

extern "C" int ps_batch_add_rollouts(ps_batch* b, const float* rollouts, int n_rows, int T, int broadcast_d,
                                     float* state_cost) {
    clear_error();
    if (!b) return set_error(PS_EINVAL, "NULL batch");
    if (n_rows <= 0 || T <= 0 || !rollouts || !state_cost) return set_error(PS_EINVAL, "empty rollouts or NULL buffer");
    if ((int)b->treq.size() >= b->lim.max_traj_requests) return set_error(PS_EINVAL, "too many trajectory requests");
    const long long n = (long long)n_rows * T;
    if ((long long)b->n_wp + b->n_roll + n > b->lim.max_waypoints)
        return set_error(PS_EINVAL, "waypoint capacity exceeded");
    b->n_roll += (int)n;
    b->treq.push_back(TrajReq{rollouts, state_cost, nullptr, nullptr, T, b->lim.max_waypoints - b->n_roll, n_rows, 1,
                              broadcast_d ? 1 : 0, 0});
    return PS_OK;
}

extern "C" int ps_batch_launch(ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep,
                               const ps_cost_params* cp, void* stream) {
    PS_NVTX("ps_batch_launch");
    clear_error();
    if (!b || !ep || !cp) return set_error(PS_EINVAL, "NULL argument");
    if (int rc = validate_scene(b->model, sv)) return rc;
    if (ep->compute_clearance) return set_error(PS_EINVAL, "batched edge checks do not compute clearance");
    if (cp->layout != PS_LAYOUT_BTD) return set_error(PS_EINVAL, "batched trajectories use PS_LAYOUT_BTD");
    cudaStream_t s = (cudaStream_t)stream;
    // the previous replay reads the pinned tables until it is done
    if (b->launched) PS_TRY_CUDA(cudaEventSynchronize(b->done));
    if (!b->ereq.empty()) std::memcpy(b->h_ereq, b->ereq.data(), sizeof(EdgeReq) * b->ereq.size());
    if (!b->treq.empty()) std::memcpy(b->h_treq, b->treq.data(), sizeof(TrajReq) * b->treq.size());
    *b->h_cnt = Counts{(int)b->ereq.size(), (int)b->treq.size(), b->n_edges, b->n_wp, b->n_roll};
    std::vector<unsigned char> key = make_key(b, sv, ep, cp);
    if (!b->exec || key != b->key) {
        b->key.clear();
        if (int rc = batch_capture(b, sv, ep, cp)) return rc;
        b->key = key;
    }
    PS_TRY_CUDA(cudaGraphLaunch(b->exec, s));
    PS_TRY_CUDA(cudaEventRecord(b->done, s));
    b->launched = true;
    return PS_OK;
}

extern "C" int ps_batch_status(ps_batch* b, int* status) {
    clear_error();
    if (!b || !status) return set_error(PS_EINVAL, "NULL argument");
    *status = PS_OK;
    if (!b->launched || b->lim.max_edges <= 0) return PS_OK;
    PS_TRY_CUDA(cudaEventSynchronize(b->done));
    EdgeWs h;
    PS_TRY_CUDA(cudaMemcpy(&h, b->d_hdr, sizeof(EdgeWs), cudaMemcpyDeviceToHost));
    *status = h.timed_out ? PS_ETIMEOUT : PS_OK;
    return PS_OK;
}

extern "C" int ps_batch_set_shape(ps_batch* b, const ps_batch_tuning* shape) {
    clear_error();
    if (!b || !shape) return set_error(PS_EINVAL, "NULL argument");
    if (!(shape->edge_share > 0.0f && shape->edge_share <= 1.0f) ||
        !(shape->traj_share > 0.0f && shape->traj_share <= 1.0f))
        return set_error(PS_EINVAL, "edge_share and traj_share must lie in (0, 1]");
    if ((shape->traj_threads != 128 && shape->traj_threads != 256) ||
        (shape->work_threads != 128 && shape->work_threads != 256))
        return set_error(PS_EINVAL, "traj_threads and work_threads must be 128 or 256");
    if (shape->layout != 0 && shape->layout != 1) return set_error(PS_EINVAL, "layout must be 0 or 1");
    if (shape->work_cost_warps < 1 || shape->work_cost_warps > shape->work_threads / 32)
        return set_error(PS_EINVAL, "work_cost_warps must be 1 .. work_threads / 32");
    b->edge_share = shape->edge_share;
    b->traj_share = shape->traj_share;
    b->traj_threads = shape->traj_threads;
    b->traj_tile = 1;
    b->layout = shape->layout;
    b->work_threads = shape->work_threads;
    b->work_cost_warps = shape->work_cost_warps;
    return PS_OK;   // the next launch captures a graph for the new shape
}

extern "C" int ps_batch_tune(ps_batch* b, const ps_scene_view* sv, const ps_edge_params* ep,
                             const ps_cost_params* cp, ps_batch_tuning* out) {
    PS_NVTX("ps_batch_tune");
    clear_error();
    if (!b) return set_error(PS_EINVAL, "NULL batch");
    const float edge_shares[] = {0.5f, 0.75f, 1.0f};
    const float traj_shares[] = {0.25f, 0.5f, 1.0f};
    const int widths[] = {128, 256};
    const int tiles[] = {1};
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, z = nullptr;
    PS_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&z) != cudaSuccess) {
        const cudaError_t le = cudaGetLastError();
        if (a) cudaEventDestroy(a);
        cudaStreamDestroy(s);
        return cuda_error(le, "tuning events");
    }
    const float keep_e = b->edge_share, keep_t = b->traj_share;
    const int keep_w = b->traj_threads, keep_tile = b->traj_tile, keep_l = b->layout, keep_k = b->work_threads,
              keep_c = b->work_cost_warps;
    float best = 3.0e38f, best_e = keep_e, best_t = keep_t;
    int best_w = keep_w, best_tile = keep_tile, best_l = keep_l, best_k = keep_k, best_c = keep_c;
    int rc = PS_OK;
    const bool edges = b->lim.max_edges > 0, trajs = b->lim.max_waypoints > 0;
    auto time_now = [&](float& ms_min) {   // capture + warm-up, then the best of 3 launches
        int r = ps_batch_launch(b, sv, ep, cp, s);
        ms_min = 3.0e38f;
        for (int k = 0; k < 3 && r == PS_OK; ++k) {
            cudaEventRecord(a, s);
            r = ps_batch_launch(b, sv, ep, cp, s);
            cudaEventRecord(z, s);
            if (cudaEventSynchronize(z) != cudaSuccess) r = cuda_error(cudaGetLastError(), "tuning run");
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, a, z);
            ms_min = std::min(ms_min, ms);
        }
        return r;
    };
    // layout 1: one work-queue kernel; (threads per block, warps that also
    // take waypoint groups)
    const int work_shapes[][2] = {{256, 8}, {256, 4}, {256, 2}, {128, 4}, {128, 2}};
    b->layout = 1;
    for (const auto& ws : work_shapes) {
        if (!trajs && ws[1] != ws[0] / 32) continue;   // no waypoints: one shape per width
        b->work_threads = ws[0];
        b->work_cost_warps = ws[1];
        float ms_min = 0.0f;
        rc = time_now(ms_min);
        if (rc) break;
        if (ms_min < best) {
            best = ms_min;
            best_l = 1;
            best_k = ws[0];
            best_c = ws[1];
        }
    }
    b->layout = 0;
    for (float es : edge_shares) {
        if (rc) break;
        if (!edges && es != 1.0f) continue;
        for (float ts : traj_shares) {
            for (int w : widths) {
                for (int tl : tiles) {
                    if (!trajs && (ts != 0.5f || w != 256 || tl != 1)) continue;
                    b->edge_share = es;
                    b->traj_share = ts;
                    b->traj_threads = w;
                    b->traj_tile = tl;
                    float ms_min = 0.0f;
                    rc = time_now(ms_min);
                    if (rc) break;
                    if (ms_min < best) {
                        best = ms_min;
                        best_l = 0;
                        best_e = es;
                        best_t = ts;
                        best_w = w;
                        best_tile = tl;
                    }
                }
                if (rc) break;
            }
            if (rc) break;
        }
        if (rc) break;
    }
    cudaStreamSynchronize(s);
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    cudaStreamDestroy(s);
    if (rc) {
        b->edge_share = keep_e;
        b->traj_share = keep_t;
        b->traj_threads = keep_w;
        b->traj_tile = keep_tile;
        b->layout = keep_l;
        b->work_threads = keep_k;
        b->work_cost_warps = keep_c;
        return rc;
    }
    b->edge_share = best_e;
    b->traj_share = best_t;
    b->traj_threads = best_w;
    b->traj_tile = best_tile;
    b->layout = best_l;
    b->work_threads = best_k;
    b->work_cost_warps = best_c;
    if (out) {
        out->edge_share = best_e;
        out->traj_share = best_t;
        out->traj_threads = best_w;
        out->traj_tile = best_tile;
        out->best_ms = best;
        out->layout = best_l;
        out->work_threads = best_k;
        out->work_cost_warps = best_c;
    }
    return PS_OK;
}
