/*
 * oracle.h -- CPU restatement of PrismPlan's collision-kinematics path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA product
 * in prismplan_b200/; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it. The product never links, calls or falls back to it.
 *
 * Every function restates a reference formula and cites the reference file
 * (paths inside code/gpu_planning/). Two precisions are provided:
 *   prec = 64 : FP64 arithmetic, libm sin/cos -- the numerical oracle
 *               (distance to contact for flipped decisions, costs, FD gradients).
 *   prec = 32 : FP32 arithmetic in the reference's operation order with
 *               std::sin/std::cos -- the multithreaded host CPU baseline.
 *
 * Parity of the FP64 FK and sphere-vs-OBB predicate is pinned against the
 * reference's own NumPy oracle (tests/test_tree_fk_vs_cpu.py:25-78) through
 * committed golden fixtures; Boolean bit-exactness of the CUDA path is pinned
 * against the reference kernels themselves (oracle/_ref, GPU tests).
 */
#ifndef PRISM_ORACLE_H
#define PRISM_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include "../include/prism_b200.h"   /* ps_model_desc / ps_scene_view layouts only */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;
typedef struct orc_scene orc_scene;

/* Build from the same descriptor the product takes (host arrays). NULL on error. */
orc_model* orc_model_create(const ps_model_desc* desc);
void       orc_model_destroy(orc_model* m);

/* Host copies of a scene in SceneCollisionData layout
   (cpp/src/collision/scene_collision_data.hh:10-47). Any array may be NULL
   when its count is 0. esdf_mode: 0 nearest (reference), 1 trilinear. */
orc_scene* orc_scene_create(const float* obb_dims, const float* obb_pose,
                            const uint8_t* obb_enable, int n_obbs,
                            const float* voxel_params, const float* voxel_pose,
                            const uint8_t* voxel_enable, const float* voxel_features,
                            int n_layers, int max_voxels_per_layer,
                            const uint8_t* sphere_acm_mask,
                            const uint8_t* sphere_obb_acm_mask,
                            const uint8_t* sphere_obb_acm_mask_approx,
                            int esdf_mode);
void       orc_scene_destroy(orc_scene* s);
/* ACM masks (sizes n_spheres*L, n_spheres*n_obbs, n_approx*n_obbs); NULL/0 = none. */
void       orc_scene_set_masks(orc_scene* s, const uint8_t* acm, int n_acm,
                               const uint8_t* obb_acm, int n_obb_acm,
                               const uint8_t* obb_acm_apx, int n_obb_acm_apx);

/* World sphere centres, out [n*n_spheres*3] (double). */
void orc_fk_spheres(const orc_model* m, const float* q, int n, int prec, double* out);

/* Configuration check (two-phase, environment; optional self).
   hit[n] u8, clearance[n] (NULL to skip) per flags (PS_CLEARANCE_*),
   gap[n] (NULL to skip): FP64 signed distance to contact of the gated exact
   pairs, min over pairs of (|c| - (r + margin)), the quantity the decision
   thresholds at 0. Returns 0. */
int orc_check_configs(const orc_model* m, const orc_scene* s, const float* q, int n,
                      float margin, unsigned flags, int prec, int threads,
                      uint8_t* hit, double* clearance, double* gap);

/* Edge checks: samples j=1..G at t=(float)j/(float)G, interpolated in FP32 as
   from + t*(to-from) with one rounding of the product-sum (edge_eval.cuh:115-121);
   when G % 16 != 0 the start configuration (the reference's padding slots,
   t = 0) is part of the verdict too.
   G[n_edges] given explicitly. valid[e], cost[e] (FLT_MAX if invalid),
   clearance[e] (NULL to skip; ESDF min like edge_eval.cuh:133-154),
   gap[e] (NULL to skip; min over samples of the sample gap).
   early_exit: stop an edge at its first colliding sample. */
int orc_check_edges(const orc_model* m, const orc_scene* s, const float* from,
                    const float* to, const int* G, int n_edges, float margin,
                    int check_self, int compute_clearance, int early_exit,
                    int prec, int threads, uint8_t* valid, double* cost,
                    double* clearance, double* gap, long long* samples_done);

/* Per-waypoint state cost w*(sum esdf hinge + sum obb hinge + self hinge)
   (chomp.cu:151-188 / stomp.cu:206-245). q is [n*n_dof]. out[n]. */
int orc_state_cost(const orc_model* m, const orc_scene* s, const float* q, int n,
                   float w, float world_margin, float self_margin, int include_self,
                   int prec, int threads, double* out);

/* Same, evaluated at an FP64 configuration (for finite differences). */
double orc_state_cost_d(const orc_model* m, const orc_scene* s, const double* q,
                        double w, double world_margin, double self_margin,
                        int include_self);

/* Distance of a configuration to the nearest kink of the state cost: hinge
   activation, min-over-OBB ties, box-region changes and self-min ties, in
   metres of the underlying clearances. Used to exclude FD-invalid points. */
double orc_state_cost_kink_distance(const orc_model* m, const orc_scene* s,
                                    const double* q, double world_margin,
                                    double self_margin, int include_self);

/* FP64 central finite-difference gradient of the state cost, h step,
   q [n*n_dof] (float inputs), grad [n*n_dof]. */
int orc_state_cost_fd_grad(const orc_model* m, const orc_scene* s, const float* q, int n,
                           float w, float world_margin, float self_margin,
                           int include_self, double h, int threads, double* grad);

/* Control-cost matrix R = dt * (A^T A) central T x T block of the 6-padded
   5-point acceleration operator (chomp_precompute.cpp:20-37), FP64, [T*T]. */
void orc_control_cost_R(int T, double delta_t, double* R);

#ifdef __cplusplus
}
#endif
#endif
