/*
 * prism_b200.h -- C ABI of the B200 (sm_100a) collision-kinematics substrate.
 *
 * This is the drop-in boundary for PrismPlan's shared collision-kinematics
 * path (code/gpu_planning/cpp/src/planning/robot_model.cuh,
 * runtime_kinematics.cuh, code/gpu_planning/cpp/src/collision/
 * scene_collision*.{cuh,hh}, two_phase_cc.cuh and the kernels that wrap them).
 *
 * Conventions
 *   - Every entry point returns an int status (PS_OK on success). On failure
 *     ps_last_error() returns a thread-local, human-readable message. No
 *     exception crosses this boundary and nothing calls exit().
 *   - Pointers documented as "device" are CUDA global-memory pointers owned by
 *     the caller. Pointers documented as "host" are plain host memory.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Every compute call is asynchronous on that stream, allocates nothing and
 *     never synchronises, so it can be captured into a CUDA graph. The
 *     optimiser loops (ps_chomp_optimize, ps_stomp_optimize) are the
 *     exception: they capture and replay their own graph and synchronise the
 *     stream between replays.
 *   - Calls on distinct streams are thread-safe: kernels use no mutable
 *     __device__ globals; all state lives in caller-owned buffers or in the
 *     immutable model object.
 *   - Joint type codes are the reference's (utils.cuh:20-26).
 */
#ifndef PRISM_B200_H
#define PRISM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define PS_OK        0
#define PS_EINVAL    1   /* bad argument, shape or capacity               */
#define PS_ENOMEM    2   /* device or host allocation failed (create only) */
#define PS_ECUDA     3   /* a CUDA runtime call or kernel launch failed    */
#define PS_ETIMEOUT  4   /* a bounded device-side wait gave up             */

/* ---- joint types (utils.cuh:20-26) ---------------------------------------- */
#define PS_FIXED   (-1)
#define PS_X_PRISM   0
#define PS_Y_PRISM   1
#define PS_Z_PRISM   2
#define PS_X_ROT     3
#define PS_Y_ROT     4
#define PS_Z_ROT     5

/* ---- limits --------------------------------------------------------------- */
#define PS_MAX_DOF       14    /* robot_model.cuh:14 (MAX_DIM)              */
#define PS_MAX_JOINTS    20    /* joint_in_collision has 20 slots per config
                                  (two_phase_cc.cuh:72, scene_collision.cuh:535) */
#define PS_MAX_SPHERES   512
#define PS_MAX_OBBS      1024
#define PS_MAX_LAYERS    8

/* Last error message of the calling thread ("" if none). */
const char* ps_last_error(void);

/* Library version string. */
const char* ps_version(void);

/* =========================================================================
 * Robot model
 * Replaces ppln::RobotModelDevice::create / destroy
 * (cpp/src/planning/robot_model.cuh:91-293) and the pybind
 * RobotModelBuilder::build_on_device / update_joint_limits / destroy
 * (cpp/src/python/bindings.cpp:118-225). Field meanings are the builder's.
 * ========================================================================= */
typedef struct ps_model_desc {
    int          n_dof;
    int          n_joints;
    const float* fixed_transforms;        /* host [n_joints*16], row-major 4x4 */
    const int*   joint_types;             /* host [n_joints]                   */
    int          n_spheres;
    const float* spheres;                 /* host [n_spheres*4] (x,y,z,r), link frame */
    const int*   sphere_to_joint;         /* host [n_spheres]                  */
    int          n_self_cc_ranges;
    const int*   self_cc_ranges;          /* host [n*3] {sphere_i, start, end}, end inclusive */
    int          n_approx_spheres;
    const float* approx_spheres;          /* host [n_approx*4]                 */
    const int*   approx_sphere_to_joint;  /* host [n_approx]                   */
    int          n_approx_self_cc_ranges;
    const int*   approx_self_cc_ranges;   /* host [n*3]                        */
    const float* approx_fixed_transforms; /* host [n_joints*16] or NULL = same as full */
    const int*   approx_joint_types;      /* host [n_joints]    or NULL = same as full */
    const float* joint_lower;             /* host [n_dof]                      */
    const float* joint_upper;             /* host [n_dof]                      */
    /* Kinematic tree; any NULL array takes the serial-chain default
       (robot_model.cuh:204-236). */
    const int*   joint_parents;           /* host [n_joints] or NULL */
    const int*   joint_id_to_dof;         /* host [n_joints] or NULL */
    const int*   t_memory_idx;            /* host [n_joints] or NULL */
    const int*   dfs_order;               /* host [n_joints] or NULL */
} ps_model_desc;

typedef struct ps_model ps_model;

typedef struct ps_model_info {
    int n_dof, n_joints, n_spheres, n_approx_spheres;
    int n_self_pairs, n_approx_self_pairs;   /* expanded (i,j) pair counts */
    int n_t_slots;
    int approx_shares_chain;                 /* 1: approx FK == full FK    */
    int device;                              /* CUDA ordinal of the upload */
    size_t device_bytes;                     /* bytes of the device blob   */
} ps_model_info;

/* Validates the descriptor, builds the kernel layout on the host and uploads
   it (one allocation, one copy) to the current CUDA device. Synchronous. */
int ps_model_create(const ps_model_desc* desc, ps_model** out);
/* Frees the device blob. Safe on NULL. */
int ps_model_destroy(ps_model* model);
/* Re-uploads joint limits without a rebuild (bindings.cpp:181-205). Host
   arrays of n_dof floats. Synchronous. The reference also re-derives
   joint_range = upper - lower; no kernel here reads a range, so none is kept. */
int ps_model_set_limits(ps_model* model, const float* lower, const float* upper);
int ps_model_get_info(const ps_model* model, ps_model_info* info);
/* Reads and clears the model's device error latch (synchronous): *code is
   PS_OK, or PS_ETIMEOUT when a kernel using this model gave up a bounded
   wait since the last poll (its outputs for that launch are incomplete).
   Replaces the reference's cudaCheckError -> exit() (utils.cuh:433-439). */
int ps_model_poll_status(ps_model* model, int* code);
/* Polls of the bounded wait with which each kernel stages this model into
   shared memory (default 2^22, far beyond a real copy; < 0 restores it).
   Takes effect for later launches (a captured graph keeps the value it was
   captured with). When a wait gives up, the kernel latches PS_ETIMEOUT
   (ps_model_poll_status) and writes fail-closed outputs: configurations in
   collision, edges invalid (cost FLT_MAX, and PS_ETIMEOUT from
   ps_edges_status / ps_batch_status on the persistent paths), costs,
   clearances and gradients NaN. With 0 every wait gives up at once, which
   is how the failure paths are tested without a fault. No reference
   counterpart (its waits are unbounded, utils.cuh:433-439). */
int ps_model_set_wait_limit(ps_model* model, int polls);

/* =========================================================================
 * Scene view: non-owning device pointers in the exact layout of
 * ppln::collision::SceneCollisionData (cpp/src/collision/scene_collision_data.hh:10-47),
 * i.e. what prrtc.SceneCollisionDataBuilder::build() produces
 * (cpp/src/python/bindings.cpp:363-402). Nothing is copied at bind time.
 * ========================================================================= */
#define PS_ESDF_NEAREST    0   /* reference lookup (scene_collision.cuh:202-331) */
#define PS_ESDF_TRILINEAR  1   /* trilinear sampling (new; no reference counterpart) */

typedef struct ps_scene_view {
    const float*   obb_dims;        /* device [n_obbs*4]  dx,dy,dz,pad (full extents) */
    const float*   obb_pose;        /* device [n_obbs*8]  inverse pose t,qw,qx,qy,qz,pad */
    const uint8_t* obb_enable;      /* device [n_obbs]    0/1 */
    int            n_obbs;
    const float*   voxel_params;    /* device [L*4] dx,dy,dz,voxel_size */
    const float*   voxel_pose;      /* device [L*8] inverse pose */
    const uint8_t* voxel_enable;    /* device [L] */
    const float*   voxel_features;  /* device [L*max_voxels_per_layer], positive = inside */
    int            n_voxel_layers;
    int            max_voxels_per_layer;
    const uint8_t* sphere_acm_mask;             /* device [n_spheres*L] or NULL */
    const uint8_t* sphere_obb_acm_mask;         /* device [n_spheres*n_obbs] or NULL */
    const uint8_t* sphere_obb_acm_mask_approx;  /* device [n_approx*n_obbs] or NULL. Read by nothing: the
                                                   reference's approximate pass passes sphere index -1 and so
                                                   applies no mask (scene_collision.cuh:584-606) */
    int            esdf_mode;       /* PS_ESDF_NEAREST or PS_ESDF_TRILINEAR */
} ps_scene_view;

/* =========================================================================
 * Batched configuration check (config-major, one lane per configuration).
 * Replaces pRRTC::check_collision_scene + check_collision_scene_kernel
 * (cpp/src/planning/pRRTC.cu:2337-2423) and prrtc.check_collision_scene
 * (cpp/src/python/bindings.cpp:493-532). The verdict is the two-phase one of
 * two_phase_cc (cpp/src/collision/two_phase_cc.cuh:57-138): approximate
 * spheres gate, per joint, the exact sphere tests.
 * ========================================================================= */
#define PS_CHECK_SELF       0x01u  /* also run the two-phase self check        */
#define PS_CLEARANCE_OBB    0x02u  /* clearance includes sphere-OBB SDF         */
#define PS_CLEARANCE_ESDF   0x04u  /* clearance includes ESDF (reference a13)   */
#define PS_NO_GATE          0x08u  /* skip the approximate gate (diagnostics)   */
/* Grid of the configuration kernel: k blocks per SM (1..15) in bits 8..11 of
   flags; 0 = 8. ps_tune_configs picks it. */
#define PS_CONFIG_BLOCKS_PER_SM(k) (((unsigned)(k) & 15u) << 8)

/* q: device [n*n_dof] row-major. hit: device [n] (1 = in collision).
   clearance: device [n] or NULL; min over spheres (radius + margin) of the
   selected clearance sources, 1000.0 when nothing is in range. */
int ps_check_configs(const ps_model* model, const ps_scene_view* scene,
                     const float* q, int n, float collision_margin,
                     unsigned flags, uint8_t* hit, float* clearance,
                     void* stream);

/* Autotuner of ps_check_configs' grid: times every blocks-per-SM choice on
   the caller's configurations (same margin, flags and outputs) and returns
   the fastest in *out and as *tuned_flags (flags with
   PS_CONFIG_BLOCKS_PER_SM set). Synchronous. No reference counterpart. */
typedef struct ps_config_tuning {
    int   blocks_per_sm;    /* the fastest grid                               */
    float best_ms;          /* median time of one call with it               */
    float default_ms;       /* same with the default grid                    */
    int   candidates;       /* grids timed                                   */
} ps_config_tuning;
int ps_tune_configs(const ps_model* model, const ps_scene_view* scene,
                    const float* q, int n, float collision_margin,
                    unsigned flags, uint8_t* hit, float* clearance,
                    void* stream, ps_config_tuning* out, unsigned* tuned_flags);

/* =========================================================================
 * Edge checks. Replaces ppln::search::evaluate_edges_batch and
 * EdgeEvalGpu::evaluate (cpp/src/planning/edge_eval.cuh:37-165,
 * cpp/src/planning/edge_batch_bridge.hh:60-96). Samples sit at t = j/G,
 * j = 1..G (the start configuration is not checked, edge_eval.cuh:110-121).
 * Outputs: valid[e] (1 = free), cost[e] = L2 length if valid else FLT_MAX,
 * clearance[e] = min ESDF clearance over the samples (only when requested;
 * FLT_MAX otherwise), exactly as edge_eval.cuh:157-164.
 * ========================================================================= */
typedef struct ps_edge_params {
    int   granularity;      /* G for every edge when samples_per_edge is NULL
                               and both rules below are off (edge_eval.cuh:38) */
    float resolution;       /* > 0: G = clamp(ceil(L2/resolution), 2, 1024)
                               (edge_eval.cuh:54-60)                            */
    float max_joint_step;   /* > 0: G = clamp(ceil(Linf/step), 1, max_samples) */
    int   max_samples;      /* clamp for the L-inf rule; <= 0 means 1024        */
    float collision_margin; /* added to every radius (edge_eval.cuh:39)         */
    int   check_self;       /* also run the self check (edge_eval.cuh:40)       */
    int   compute_clearance;/* ESDF min clearance over samples (edge_eval.cuh:41) */
    float time_budget_ms;   /* > 0: persistent paths (ps_check_edges,
                               ps_check_edges_static, ps_batch) stop pulling
                               work once this much device time has passed
                               since the call's first kernel began; edges left
                               unfinished come back invalid (cost FLT_MAX)
                               and the status query reports PS_ETIMEOUT. The
                               planners' own device deadline is the model
                               (pRRTC.cu:1595-1602). 0: no limit. The plain
                               path ignores it. No reference field.          */
    /* Launch shape of the persistent paths; 0 = automatic, and
       ps_tune_edges picks them. No reference fields. */
    int   probe;            /* end-sample probe: 0 automatic (on with at least
                               8 warps of edges per SM, boxes-only scenes),
                               1 on (boxes-only scenes), 2 off              */
    int   queue_blocks_per_sm; /* resident queue blocks per SM: 0 = all that
                               fit, k > 0 = at most k                       */
    int   grab;             /* queue items a warp takes per grab: 0 =
                               automatic (up to 32), 1..32 fixed            */
} ps_edge_params;

/* Plain per-call path: one warp per edge, samples in order, early exit at the
   first colliding sample. samples_per_edge: device [n_edges] or NULL. */
int ps_check_edges_plain(const ps_model* model, const ps_scene_view* scene,
                         const float* from, const float* to,
                         const int* samples_per_edge, int n_edges,
                         const ps_edge_params* params,
                         uint8_t* valid, float* cost, float* clearance,
                         void* stream);

/* Device workspace the persistent edge path needs (caller allocates). */
size_t ps_edges_workspace_bytes(int n_edges);

/* Persistent work-queue path: edges are cut into warp-sized sample chunks,
   ordered chunk-major and pulled from a global queue by a persistent grid;
   an edge found in collision retires its remaining chunks. All launches are
   capture-safe. workspace: device, >= ps_edges_workspace_bytes(n_edges). */
int ps_check_edges(const ps_model* model, const ps_scene_view* scene,
                   const float* from, const float* to,
                   const int* samples_per_edge, int n_edges,
                   const ps_edge_params* params,
                   uint8_t* valid, float* cost, float* clearance,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Persistent edge checks with the workspace built into the library, for
   callers that cannot allocate device memory: a planner evaluating an edge
   batch per search expansion cannot afford cudaMalloc/cudaFree inside its
   latency budget (both can synchronise the device), and some host processes
   have no CUDA allocator of their own to provide a workspace from. No
   counterpart in the reference (its EdgeEvalGpu owns cudaMalloc'd buffers).
   Same arguments, verdicts and outputs as ps_check_edges minus the
   workspace. Limits and sharing:
     - n_edges <= PS_EDGES_STATIC_MAX (65536); larger batches return PS_EINVAL.
       The scratch array (about 1.5 MiB) is a file-scope __device__ array, held
       by every GPU that loads the library until the process exits.
     - The first call on each device looks up the array's device address
       (cudaGetSymbolAddress) with that device current; make that first call
       before any stream capture on the device. The address is kept for the
       life of the process: after cudaDeviceReset on a device, this entry
       point must not be called again on it (the kept address belongs to
       the destroyed context).
     - Every call on a device shares the one array and resets it as it starts,
       so calls whose work overlaps on the GPU (other streams or threads) race.
   Allocates nothing: no cudaMalloc, cudaFree or allocating library call. */
#define PS_EDGES_STATIC_MAX 65536
int ps_check_edges_static(const ps_model* model, const ps_scene_view* scene,
                          const float* from, const float* to,
                          const int* samples_per_edge, int n_edges,
                          const ps_edge_params* params,
                          uint8_t* valid, float* cost, float* clearance,
                          void* stream);

/* Autotuner of the persistent edge path (ps_check_edges). Times every
   candidate launch shape -- probe on and off, queue residency from all that
   fit down by two blocks per SM, grab sizes automatic / 8 / 32 -- on the
   caller's edges and writes the fastest to *tuned (a copy of *params with
   probe, queue_blocks_per_sm and grab set; pass it to later calls on edges of
   that kind and count) and to *out. Verdicts and costs do not depend on the
   shape. Synchronous; runs ps_check_edges several times on `stream` with the
   caller's buffers. No reference counterpart. */
typedef struct ps_edge_tuning {
    int   probe, queue_blocks_per_sm, grab;   /* the fastest shape            */
    float best_ms;          /* median time of one call with it               */
    float default_ms;       /* same with every shape field 0                 */
    int   candidates;       /* shapes timed                                  */
} ps_edge_tuning;
int ps_tune_edges(const ps_model* model, const ps_scene_view* scene,
                  const float* from, const float* to,
                  const int* samples_per_edge, int n_edges,
                  const ps_edge_params* params,
                  uint8_t* valid, float* cost, float* clearance,
                  void* workspace, size_t workspace_bytes, void* stream,
                  ps_edge_tuning* out, ps_edge_params* tuned);

/* Status of the last persistent call that used `workspace` (NULL: the
   built-in workspace of the current device): PS_OK, or PS_ETIMEOUT when its
   time budget ran out. Synchronous (reads the workspace header). */
int ps_edges_status(const void* workspace, int* status);

/* Host-buffer edge bridge. Replaces ppln::search::EdgeEvalGpu
   (cpp/src/planning/edge_batch_bridge.hh:27-111): the object owns device
   buffers for max_edges edges, pinned host mirrors, the persistent path's
   workspace and a private stream, all allocated at create.
     ps_edge_bridge_create   <- EdgeEvalGpu(dim, max_edges, scene, model)
                                (:29-45); dim must equal the model's n_dof.
                                The scene view is copied (its device pointers
                                must stay valid); ps_edge_bridge_set_scene
                                replaces it.
     ps_edge_bridge_evaluate <- EdgeEvalGpu::evaluate (:60-96): from_flat /
                                to_flat are HOST row-major [num_edges * dim];
                                out_valid / out_cost (and out_clearance when
                                params->compute_clearance) are HOST arrays of
                                num_edges. Synchronous, like the reference:
                                stage into the pinned mirrors, copy in, check
                                (ps_check_edges, replayed from a CUDA graph per
                                edge count, parameters and scene), copy out,
                                synchronise. The staging runs in slices and
                                each slice's copy starts as soon as it is
                                staged; inputs already in the bridge's own
                                mirrors (ps_edge_bridge_host_inputs) are not
                                staged. num_edges <= 0: nothing to do, PS_OK;
                                num_edges > max_edges: PS_EINVAL (the
                                reference throws, :67-68).
     ps_edge_bridge_status   <- PS_ETIMEOUT when the time budget of the call
                                waited for last ran out (ps_edges_status of
                                its workspace).
     ps_edge_bridge_destroy  <- ~EdgeEvalGpu (:47-53).
   One bridge per host thread at a time, on the device that was current at
   create (evaluate returns PS_EINVAL on another). */
typedef struct ps_edge_bridge ps_edge_bridge;
#define PS_BRIDGE_SLOTS 2
int ps_edge_bridge_create(const ps_model* model, const ps_scene_view* scene,
                          int dim, int max_edges, ps_edge_bridge** out);
int ps_edge_bridge_set_scene(ps_edge_bridge* bridge, const ps_scene_view* scene);
int ps_edge_bridge_evaluate(ps_edge_bridge* bridge, const float* from_flat,
                            const float* to_flat, int num_edges,
                            const ps_edge_params* params, uint8_t* out_valid,
                            float* out_cost, float* out_clearance);
/* Asynchronous form, no reference counterpart: up to PS_BRIDGE_SLOTS calls
   in flight, one per slot, each with its own buffers and stream, so that a
   caller can stage and copy in one batch while the GPU checks another.
   ps_edge_bridge_submit stages the host edges into the slot's pinned mirror
   (the caller's arrays may be reused once it returns) and queues the copy
   in, the check and the copy out; ps_edge_bridge_wait waits for that slot's
   call and writes its outputs to host arrays (out_clearance when the call's
   params asked for clearance). A slot takes a new call only after the
   previous one was waited for (PS_EINVAL otherwise). ps_edge_bridge_evaluate
   is submit + wait on slot 0. ps_edge_bridge_status reports the call waited
   for last. */
int ps_edge_bridge_submit(ps_edge_bridge* bridge, int slot, const float* from_flat,
                          const float* to_flat, int num_edges,
                          const ps_edge_params* params);
int ps_edge_bridge_wait(ps_edge_bridge* bridge, int slot, uint8_t* out_valid,
                        float* out_cost, float* out_clearance);
int ps_edge_bridge_status(const ps_edge_bridge* bridge, int* status);
/* The bridge's pinned host input mirrors of slot 0 (row-major
   [max_edges * dim] each), valid until destroy. A caller may write its edges there and pass
   these two pointers to ps_edge_bridge_evaluate, which then skips its staging
   copy. No reference counterpart (its mirrors are private). */
int ps_edge_bridge_host_inputs(ps_edge_bridge* bridge, float** from_flat, float** to_flat);
int ps_edge_bridge_destroy(ps_edge_bridge* bridge);

/* =========================================================================
 * Trajectory cost: summed hinge + self hinge + smoothness, with its exact
 * gradient from a hand-written adjoint.
 * Forward cost replaces chomp_state_cost_kernel / stomp_state_cost_kernel
 * (cpp/src/planning/chomp.cu:151-188, cpp/src/planning/stomp.cu:206-245) over
 * scene_sum_{esdf,obb}_hinge_runtime + self_min_hinge_runtime
 * (cpp/src/collision/scene_collision.cuh:394-495,
 * cpp/src/planning/runtime_kinematics.cuh:295-330); the gradient replaces the
 * central-difference chomp_obs_grad_kernel (cpp/src/planning/chomp.cu:83-144);
 * the smoothness term replaces chomp_control_cost_kernel
 * (cpp/src/planning/chomp.cu:196-210) with R from
 * cpp/src/planning/chomp_precompute.cpp:20-37 applied as a banded stencil.
 * ========================================================================= */
#define PS_MAX_TRAJ_LEN 16384  /* longest trajectory with a smoothness term */
#define PS_LAYOUT_BTD  0   /* q[b][t][d]  (torch-natural)                        */
#define PS_LAYOUT_BDT  1   /* q[b][d][t]  (reference theta[d*T+t], rollouts[(r*D+d)*T+t]) */

typedef struct ps_cost_params {
    float collision_cost_weight; /* w (CHOMP_settings.hh:35)                     */
    float world_margin;          /* hinge band eps (CHOMP_settings.hh:42)        */
    float self_margin;           /* self hinge band (CHOMP_settings.hh:43)       */
    int   include_self;          /* add self_min_hinge                            */
    float smoothness_weight;     /* lambda on theta^T R theta; 0 = off            */
    float delta_t;               /* R time step (CHOMP_settings.hh:46)            */
    int   layout;                /* PS_LAYOUT_BTD or PS_LAYOUT_BDT                */
} ps_cost_params;

/* q: device [B*T*D] in `layout`. Outputs (each device, NULL to skip):
     waypoint_cost [B*T]  = w * (sum esdf hinge + sum obb hinge + self hinge)
     traj_cost     [B]    = sum_t waypoint_cost + lambda * sum_d theta_d^T R theta_d
     grad          [B*T*D] in `layout` = d traj_cost / d q (exact adjoint).
   The collision hinge uses the full sphere set without the approximate gate,
   as the reference cost kernels do. */
int ps_traj_cost(const ps_model* model, const ps_scene_view* scene,
                 const float* q, int B, int T, const ps_cost_params* params,
                 float* waypoint_cost, float* traj_cost, float* grad,
                 void* stream);

/* STOMP rollout costs: per (rollout, waypoint) state cost over
   rollouts device [n_rows*D*T] (PS_LAYOUT_BDT, the reference layout) or
   [n_rows*T*D] (PS_LAYOUT_BTD). state_cost: device [n_rows*T]; when
   broadcast_d != 0 it is [n_rows*D*T] with the value repeated over d, as
   stomp_state_cost_kernel writes it (stomp.cu:241-244). */
int ps_rollout_costs(const ps_model* model, const ps_scene_view* scene,
                     const float* rollouts, int n_rows, int T,
                     const ps_cost_params* params, int broadcast_d,
                     float* state_cost, void* stream);

/* =========================================================================
 * Mixed-request batches: many edge-check requests of uneven length, many
 * trajectory cost+gradient requests and STOMP rollout-cost requests
 * evaluated by one CUDA-graph launch.
 * Replaces the reference's one-launch-and-sync-per-request pattern
 * (EdgeEvalGpu::evaluate, cpp/src/planning/edge_batch_bridge.hh:60-96; the
 * CHOMP iteration loop, cpp/src/planning/chomp.cu:508-555; the STOMP rollout
 * cost launch, cpp/src/planning/stomp.cu:206-245). No reference counterpart
 * for the batching itself.
 *
 * Requests hold caller device pointers; nothing is copied until launch. The
 * first launch (and any launch whose scene/params/tuning differ from the
 * last) captures the graph; later launches replay it with the new request
 * table, so a planner can re-fill and launch every iteration without
 * re-capture. Results equal the per-request calls bit for bit:
 *   edges        == ps_check_edges / ps_check_edges_plain (valid, cost);
 *   trajectories == ps_traj_cost(B=1, PS_LAYOUT_BTD) (waypoint_cost,
 *                   traj_cost, grad).
 * ps_batch_create allocates the packed device buffers and pinned host
 * tables; ps_batch_launch allocates nothing. A launch waits (host) for the
 * previous launch of the same batch before it rewrites the request table.
 * ========================================================================= */
typedef struct ps_batch ps_batch;

typedef struct ps_batch_limits {
    int max_edge_requests;   /* requests of edge checks                       */
    int max_edges;           /* total edges over all edge requests            */
    int max_traj_requests;   /* trajectory requests                           */
    int max_waypoints;       /* total waypoints over all trajectory requests  */
    int max_traj_len;        /* longest trajectory, <= PS_MAX_TRAJ_LEN        */
} ps_batch_limits;

typedef struct ps_batch_tuning {
    float edge_share;        /* fraction of the edge kernel's resident-block
                                slots its persistent grid takes              */
    float traj_share;        /* same for the trajectory kernel's grid         */
    int   traj_threads;      /* threads per block of the trajectory kernel
                                (128 or 256; 4 lanes per waypoint)           */
    int   traj_tile;         /* kept in the record; always 1                  */
    float best_ms;           /* measured time of one launch at this choice    */
    int   layout;            /* 0: the persistent edge queue and the waypoint
                                kernel run side by side in two graph branches;
                                1: one persistent work-queue kernel pulls
                                edge chunks and waypoint groups (trajectories
                                and rollouts) from global counters          */
    int   work_threads;      /* threads per block of that kernel (128, 256)  */
    int   work_cost_warps;   /* warps per block of it that also take waypoint
                                groups (1 .. work_threads / 32); fewer leave
                                shared memory for more resident blocks     */
} ps_batch_tuning;

int ps_batch_create(const ps_model* model, const ps_batch_limits* limits,
                    ps_batch** out);
int ps_batch_destroy(ps_batch* batch);
/* Forget every request (buffers stay allocated). */
int ps_batch_clear(ps_batch* batch);
/* n edges from[n*D] -> to[n*D] (device). samples: device [n] or NULL (the
   launch's ps_edge_params rule). Outputs valid[n], cost[n] (device). */
int ps_batch_add_edges(ps_batch* batch, const float* from, const float* to,
                       const int* samples, int n, uint8_t* valid, float* cost);
/* One trajectory q[T*D] (device, waypoint-major). Outputs (device, each may
   be NULL): waypoint_cost[T], traj_cost[1], grad[T*D]. A request with only
   waypoint_cost is a STOMP rollout. */
int ps_batch_add_trajectory(ps_batch* batch, const float* q, int T,
                            float* waypoint_cost, float* traj_cost, float* grad);
/* n_rows STOMP rollouts of T waypoints (device, the reference layout
   rollouts[(r*D + d)*T + t], stomp.cu:206-245). Output (device): state_cost
   [n_rows*T], or [n_rows*D*T] with each value repeated over d when
   broadcast_d != 0, as stomp_state_cost_kernel writes it. Equal to
   ps_rollout_costs bit for bit; no gradient is computed. Counts one
   trajectory request and n_rows*T waypoints of the capacity. */
int ps_batch_add_rollouts(ps_batch* batch, const float* rollouts, int n_rows, int T,
                          int broadcast_d, float* state_cost);
/* Evaluates every request. params->compute_clearance must be 0 and
   cost->layout PS_LAYOUT_BTD. */
int ps_batch_launch(ps_batch* batch, const ps_scene_view* scene,
                    const ps_edge_params* params, const ps_cost_params* cost,
                    void* stream);
/* Autotuner: times every candidate split of the SMs between the edge and the
   trajectory branch, every trajectory block width and tile size on the
   batch's current requests, keeps the fastest for later launches and
   reports it (out may be NULL). Synchronous; launches the batch several
   times. */
/* Use this launch shape from the next launch on (for example one that
   ps_batch_tune returned earlier); best_ms and traj_tile are ignored.
   Shares in (0, 1], thread counts 128 or 256, layout 0 or 1,
   work_cost_warps 1 .. work_threads / 32. */
int ps_batch_set_shape(ps_batch* batch, const ps_batch_tuning* shape);
int ps_batch_tune(ps_batch* batch, const ps_scene_view* scene,
                  const ps_edge_params* params, const ps_cost_params* cost,
                  ps_batch_tuning* out);
/* Status of the batch's last launch (waits for it): PS_OK, or PS_ETIMEOUT
   when params->time_budget_ms ran out in its edge branch. */
int ps_batch_status(ps_batch* batch, int* status);

/* =========================================================================
 * Batched CHOMP optimisation: B trajectories advance together on the
 * device. Replaces the per-request host loop of CHOMP::solve_runtime_scene
 * (cpp/src/planning/chomp.cu:358-600) with the same iteration semantics:
 *   theta <- clamp(theta - step_size (R + 1e-8 I)^-1 (obs_grad + lambda R theta))
 *   on the interior waypoints (chomp_update_kernel, chomp.cu:259-289), where
 *   obs_grad is the exact adjoint of the summed hinge (ps_traj_cost) instead
 *   of the reference's central differences (chomp.cu:71-120);
 *   total cost = sum of waypoint costs + lambda theta^T R theta
 *   (chomp.cu:196-243);
 *   validity = every waypoint and every segment sample theta_t + s/n_sub
 *   (theta_t+1 - theta_t), n_sub = ceil(max segment L2 / collision_check_step),
 *   two-phase check (chomp.cu:296-349, 459-485);
 *   best valid snapshot, num_iterations_after_valid polishing iterations and
 *   a two-iteration convergence streak below convergence_eps
 *   (chomp.cu:487-537).
 * ========================================================================= */
typedef struct ps_chomp_params {
    int   num_iterations;             /* CHOMP_settings.hh:26 (100)          */
    int   num_iterations_after_valid; /* CHOMP_settings.hh:27 (5)            */
    float step_size;                  /* CHOMP_settings.hh:33 (0.3)          */
    float smoothness_weight;          /* lambda, CHOMP_settings.hh:34 (1.0)  */
    float collision_cost_weight;      /* CHOMP_settings.hh:35 (20)           */
    float world_margin;               /* CHOMP_settings.hh:42 (0.02)         */
    float self_margin;                /* CHOMP_settings.hh:43 (0.01)         */
    float delta_t;                    /* CHOMP_settings.hh:46 (0.1)          */
    float convergence_eps;            /* CHOMP_settings.hh:49 (1e-4)         */
    float collision_check_step;       /* CHOMP_settings.hh:55 (0.05)         */
    float collision_margin;           /* validity radius margin (pRRTC_settings) */
    int   include_self;               /* self hinge in the cost (1)          */
    int   check_self;                 /* self check in the validity (1, as
                                         chomp.cu:345)                       */
    float time_limit_ms;              /* > 0: a trajectory stops iterating once
                                         this much device time has passed
                                         since the call began (chomp.cu:501-505
                                         measures host wall time). 0: none.  */
} ps_chomp_params;

/* Device workspace for ps_chomp_optimize (caller allocates, 256-byte
   aligned). 0 when the model is NULL or T < 2. */
size_t ps_chomp_workspace_bytes(const ps_model* model, int B, int T);

/* theta: device [B*T*D] (waypoint-major per trajectory), the initial
   trajectories in, the last iterate out; waypoints 0 and T-1 stay fixed.
   Outputs (device): best [B*T*D] = best valid iterate (the last iterate
   when none was valid), solved [B] (1 = a valid iterate was found),
   iterations [B] (updates applied, chomp.cu:522), best_cost [B] (total cost
   of best). 2 <= T <= 1024. Synchronises the stream every 8 iterations to
   stop once every trajectory has finished; not capturable. */
int ps_chomp_optimize(const ps_model* model, const ps_scene_view* scene,
                      float* theta, int B, int T, const ps_chomp_params* params,
                      float* best, uint8_t* solved, int* iterations,
                      float* best_cost, void* workspace, size_t workspace_bytes,
                      void* stream);

/* =========================================================================
 * Batched STOMP optimisation: B trajectories advance together on the
 * device. Replaces the per-request host loop of STOMP::solve_runtime_scene
 * (cpp/src/planning/stomp.cu:565-965) with its iteration semantics
 * (stomp.cu:786-889):
 *   rollouts: num_rollouts_new fresh noisy copies of the optimum
 *   (theta + L z, endpoints pinned, clamped; all num_rollouts_new +
 *   num_rollouts_old fresh on the first iteration), the num_rollouts_old
 *   lowest-cost rollouts of the previous iteration, and the optimum itself;
 *   per-rollout cost = state cost (the summed hinge of ps_rollout_costs) +
 *   control_cost_weight theta_d^T R theta_d;
 *   per (d, t) weights p_r = exp(-h (c_r - min) / (max - min)) / sum;
 *   theta <- theta + M (sum_r p_r noise_r), endpoints pinned, unconditionally;
 *   validity, best valid snapshot, polish budget and convergence streak as
 *   in CHOMP.
 * L L^T = (R + 1e-8 I)^-1 rescaled to max entry 1/T (times noise_scale) and
 * M = (R + 1e-8 I)^-1 with columns scaled to max 1/T (stomp_precompute.cpp:
 * 46-98) are applied as banded triangular solves with the factor of
 * R + 1e-8 I: L = sqrt(c) J (Lb^-T) J and M x = (R + 1e-8 I)^-1 (s .* x),
 * in FP64. The normal variates z come from Philox4x32-10 (Salmon et al.,
 * SC 2011) keyed by `seed` with counter (t / 4, rollout * D + d, iteration),
 * through Box-Muller: every request of a batch draws the same stream, as
 * every reference solve draws its fixed seed (stomp.cu:707), so a request's
 * result does not depend on the batch it is in. The reference draws from
 * cuRAND XORWOW; the streams differ, the distribution is the same.
 * ========================================================================= */
typedef struct ps_stomp_params {
    int   num_iterations;             /* STOMP_settings.hh (20)               */
    int   num_iterations_after_valid; /* (3)                                  */
    int   num_rollouts_new;           /* (30)                                 */
    int   num_rollouts_old;           /* (20)                                 */
    float delta_t;                    /* R time step (0.1)                    */
    float control_cost_weight;        /* (0.1)                                */
    float collision_cost_weight;      /* (20)                                 */
    float exponentiated_cost_sensitivity; /* h (2.0)                          */
    float world_margin;               /* world hinge band (0.02)              */
    float self_margin;                /* self hinge band (0.01)               */
    float convergence_eps;            /* (1e-4)                               */
    float noise_scale;                /* factor on L (1.0)                    */
    float collision_check_step;       /* validity densification (0.05)        */
    float collision_margin;           /* validity radius margin (0)           */
    int   include_self;               /* self hinge in the state cost (1)     */
    int   check_self;                 /* self check in the validity (1)       */
    float time_limit_ms;              /* > 0: device-time limit, 0: none      */
    unsigned long long seed;          /* Philox key (reference seed 0x5be5)   */
} ps_stomp_params;

/* Device workspace for ps_stomp_optimize (caller allocates, 256-byte
   aligned). 0 for invalid arguments. */
size_t ps_stomp_workspace_bytes(const ps_model* model, int B, int T,
                                const ps_stomp_params* params);

/* Same arguments and outputs as ps_chomp_optimize: theta [B*T*D] device,
   initial trajectories in, last iterate out (waypoints 0 and T-1 fixed);
   best, solved, iterations, best_cost as there. 3 <= T <= 1024;
   num_rollouts_new >= 1, num_rollouts_old >= 0, their sum + 1 <= 1024.
   Synchronises the stream every 8 iterations; not capturable. */
int ps_stomp_optimize(const ps_model* model, const ps_scene_view* scene,
                      float* theta, int B, int T, const ps_stomp_params* params,
                      float* best, uint8_t* solved, int* iterations,
                      float* best_cost, void* workspace, size_t workspace_bytes,
                      void* stream);

/* Where the last iteration's rollouts sit inside the workspace (byte
   offsets; diagnostics and tests). Rows are rollout-major over requests:
   row = r * B + b, r = 0..rows-1 (new, then old, then the optimum). Each
   iteration writes buffer (iteration & 1) of the double-buffered arrays. */
typedef struct ps_stomp_layout {
    int    rows;             /* num_rollouts_new + num_rollouts_old + 1      */
    size_t rollouts[2];      /* float [rows*B][T][D]                         */
    size_t noise;            /* float [rows*B][T][D], rollout - optimum      */
    size_t state_cost[2];    /* float [rows*B][T]                            */
    size_t row_total[2];     /* float [rows*B]: sum of state + control cost  */
    size_t reuse_index;      /* int [B][num_rollouts_old]: rows reused       */
} ps_stomp_layout;
int ps_stomp_workspace_layout(const ps_model* model, int B, int T,
                              const ps_stomp_params* params, ps_stomp_layout* out);

/* =========================================================================
 * Diagnostics
 * ========================================================================= */
/* World-frame sphere centres for n configurations (device out [n*n_spheres*3],
   sphere order as in the descriptor). Same arithmetic as the checks. */
int ps_fk_spheres(const ps_model* model, const float* q, int n,
                  float* sphere_xyz, void* stream);

/* Sphere-vs-box pairs decided exactly as the kernels decide them (3x3 fast
   path, guard band, the reference sequence of sphere_single_obb_collision,
   scene_collision.cuh:24-78, inside the band), one pair per index i:
   obb_dims [n*4], obb_pose [n*8] (SceneCollisionData layout), spheres
   [n*4] (x, y, z, radius incl. margin), all device and 16-byte aligned.
   decision [n] (device): bit 0 = hit, bit 1 = the pair fell inside the
   guard band and was re-decided with the reference sequence. local_xyz
   [n*3] (device, may be NULL): the reference sequence's box-frame
   coordinates (transform_sphere_to_local). Diagnostics and parity tests. */
int ps_debug_obb_pairs(const float* obb_dims, const float* obb_pose, const float* spheres, int n,
                       uint8_t* decision, float* local_xyz, void* stream);

/* FP32 FMA throughput probe used as the roofline denominator: 8 independent
   FMA chains per thread on every SM; returns FLOP/s (host). Synchronous; the
   only entry point besides ps_model_create that allocates (4 bytes). */
int ps_probe_fp32_peak(double* flops_per_s, void* stream);

/* Executed-work counters for roofline accounting: when dev_counters (device,
   8 x uint64) is non-NULL, every later launch adds [pair tests, exact
   re-decisions, samples, FK joint steps, sphere transforms, self pairs, ESDF
   lookups, broad-phase box tests]. Process-wide, not thread-safe; NULL
   (the default) disables counting. No reference counterpart. */
int ps_set_stats(unsigned long long* dev_counters);

/* Kernel timing hook: when both are non-NULL (cudaEvent_t as void*), each
   ps_check_configs / ps_check_edges / ps_check_edges_plain / ps_traj_cost /
   ps_rollout_costs call records `start` immediately before and `stop`
   immediately after its main kernel, on the call's stream (also inside a
   captured graph). Process-wide, not thread-safe; NULL disables. */
int ps_set_timing_events(void* start, void* stop);

#ifdef __cplusplus
}
#endif

#endif /* PRISM_B200_H */
