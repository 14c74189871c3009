"""ctypes binding of the C ABI declared in include/prism_b200.h.

The product path has exactly one implementation: the sm_100a CUDA library
``prismplan_b200/libprism_b200.so``. If it is missing or fails to load, every
entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libprism_b200.so"

PS_OK, PS_EINVAL, PS_ENOMEM, PS_ECUDA, PS_ETIMEOUT = 0, 1, 2, 3, 4
_STATUS_NAMES = {1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "ETIMEOUT"}

PS_CHECK_SELF = 0x01
PS_CLEARANCE_OBB = 0x02
PS_CLEARANCE_ESDF = 0x04
PS_NO_GATE = 0x08


def PS_CONFIG_BLOCKS_PER_SM(k):
    return (int(k) & 15) << 8


PS_ESDF_NEAREST = 0
PS_ESDF_TRILINEAR = 1
PS_LAYOUT_BTD = 0
PS_LAYOUT_BDT = 1

PS_MAX_DOF = 14
PS_MAX_JOINTS = 20
PS_MAX_SPHERES = 512
PS_MAX_OBBS = 1024
PS_MAX_LAYERS = 8
PS_EDGES_STATIC_MAX = 65536
PS_BRIDGE_SLOTS = 2
PS_MAX_TRAJ_LEN = 16384

# joint types (utils.cuh:20-26)
PS_FIXED = -1
PS_X_PRISM, PS_Y_PRISM, PS_Z_PRISM = 0, 1, 2
PS_X_ROT, PS_Y_ROT, PS_Z_ROT = 3, 4, 5


class PrismError(RuntimeError):
    """A C-ABI call returned a non-OK status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{_STATUS_NAMES.get(status, status)}] {message}")
        self.status = status


_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)


class ModelDesc(C.Structure):
    """ps_model_desc (host arrays)."""

    _fields_ = [
        ("n_dof", C.c_int), ("n_joints", C.c_int),
        ("fixed_transforms", _fp), ("joint_types", _ip),
        ("n_spheres", C.c_int), ("spheres", _fp), ("sphere_to_joint", _ip),
        ("n_self_cc_ranges", C.c_int), ("self_cc_ranges", _ip),
        ("n_approx_spheres", C.c_int), ("approx_spheres", _fp),
        ("approx_sphere_to_joint", _ip),
        ("n_approx_self_cc_ranges", C.c_int), ("approx_self_cc_ranges", _ip),
        ("approx_fixed_transforms", _fp), ("approx_joint_types", _ip),
        ("joint_lower", _fp), ("joint_upper", _fp),
        ("joint_parents", _ip), ("joint_id_to_dof", _ip),
        ("t_memory_idx", _ip), ("dfs_order", _ip),
    ]


class ModelInfo(C.Structure):
    _fields_ = [
        ("n_dof", C.c_int), ("n_joints", C.c_int), ("n_spheres", C.c_int),
        ("n_approx_spheres", C.c_int), ("n_self_pairs", C.c_int),
        ("n_approx_self_pairs", C.c_int), ("n_t_slots", C.c_int),
        ("approx_shares_chain", C.c_int), ("device", C.c_int),
        ("device_bytes", C.c_size_t),
    ]


class SceneView(C.Structure):
    """ps_scene_view (device pointers, SceneCollisionData layout)."""

    _fields_ = [
        ("obb_dims", C.c_void_p), ("obb_pose", C.c_void_p), ("obb_enable", C.c_void_p),
        ("n_obbs", C.c_int),
        ("voxel_params", C.c_void_p), ("voxel_pose", C.c_void_p),
        ("voxel_enable", C.c_void_p), ("voxel_features", C.c_void_p),
        ("n_voxel_layers", C.c_int), ("max_voxels_per_layer", C.c_int),
        ("sphere_acm_mask", C.c_void_p), ("sphere_obb_acm_mask", C.c_void_p),
        ("sphere_obb_acm_mask_approx", C.c_void_p),
        ("esdf_mode", C.c_int),
    ]


class EdgeParams(C.Structure):
    _fields_ = [
        ("granularity", C.c_int), ("resolution", C.c_float),
        ("max_joint_step", C.c_float), ("max_samples", C.c_int),
        ("collision_margin", C.c_float), ("check_self", C.c_int),
        ("compute_clearance", C.c_int), ("time_budget_ms", C.c_float),
        ("probe", C.c_int), ("queue_blocks_per_sm", C.c_int), ("grab", C.c_int),
    ]


class EdgeTuning(C.Structure):
    _fields_ = [
        ("probe", C.c_int), ("queue_blocks_per_sm", C.c_int), ("grab", C.c_int),
        ("best_ms", C.c_float), ("default_ms", C.c_float), ("candidates", C.c_int),
    ]


class ConfigTuning(C.Structure):
    _fields_ = [
        ("blocks_per_sm", C.c_int), ("best_ms", C.c_float), ("default_ms", C.c_float), ("candidates", C.c_int),
    ]


class CostParams(C.Structure):
    _fields_ = [
        ("collision_cost_weight", C.c_float), ("world_margin", C.c_float),
        ("self_margin", C.c_float), ("include_self", C.c_int),
        ("smoothness_weight", C.c_float), ("delta_t", C.c_float),
        ("layout", C.c_int),
    ]


class BatchLimits(C.Structure):
    _fields_ = [
        ("max_edge_requests", C.c_int), ("max_edges", C.c_int),
        ("max_traj_requests", C.c_int), ("max_waypoints", C.c_int),
        ("max_traj_len", C.c_int),
    ]


class BatchTuning(C.Structure):
    _fields_ = [
        ("edge_share", C.c_float), ("traj_share", C.c_float),
        ("traj_threads", C.c_int), ("traj_tile", C.c_int), ("best_ms", C.c_float),
        ("layout", C.c_int), ("work_threads", C.c_int), ("work_cost_warps", C.c_int),
    ]


class ChompParams(C.Structure):
    _fields_ = [
        ("num_iterations", C.c_int), ("num_iterations_after_valid", C.c_int),
        ("step_size", C.c_float), ("smoothness_weight", C.c_float),
        ("collision_cost_weight", C.c_float), ("world_margin", C.c_float),
        ("self_margin", C.c_float), ("delta_t", C.c_float),
        ("convergence_eps", C.c_float), ("collision_check_step", C.c_float),
        ("collision_margin", C.c_float), ("include_self", C.c_int),
        ("check_self", C.c_int), ("time_limit_ms", C.c_float),
    ]


class StompParams(C.Structure):
    _fields_ = [
        ("num_iterations", C.c_int), ("num_iterations_after_valid", C.c_int),
        ("num_rollouts_new", C.c_int), ("num_rollouts_old", C.c_int),
        ("delta_t", C.c_float), ("control_cost_weight", C.c_float),
        ("collision_cost_weight", C.c_float), ("exponentiated_cost_sensitivity", C.c_float),
        ("world_margin", C.c_float), ("self_margin", C.c_float),
        ("convergence_eps", C.c_float), ("noise_scale", C.c_float),
        ("collision_check_step", C.c_float), ("collision_margin", C.c_float),
        ("include_self", C.c_int), ("check_self", C.c_int),
        ("time_limit_ms", C.c_float), ("seed", C.c_ulonglong),
    ]


class StompLayout(C.Structure):
    _fields_ = [
        ("rows", C.c_int), ("rollouts", C.c_size_t * 2), ("noise", C.c_size_t),
        ("state_cost", C.c_size_t * 2), ("row_total", C.c_size_t * 2), ("reuse_index", C.c_size_t),
    ]


# (name, restype, argtypes)
_SIGNATURES = [
    ("ps_last_error", C.c_char_p, []),
    ("ps_version", C.c_char_p, []),
    ("ps_model_create", C.c_int, [C.POINTER(ModelDesc), C.POINTER(C.c_void_p)]),
    ("ps_model_destroy", C.c_int, [C.c_void_p]),
    ("ps_model_set_limits", C.c_int, [C.c_void_p, _fp, _fp]),
    ("ps_model_get_info", C.c_int, [C.c_void_p, C.POINTER(ModelInfo)]),
    ("ps_model_poll_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("ps_model_set_wait_limit", C.c_int, [C.c_void_p, C.c_int]),
    ("ps_tune_edges", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                C.c_void_p, C.c_void_p]),
    ("ps_tune_configs", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_uint, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_debug_obb_pairs", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    ("ps_check_configs", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_int, C.c_float, C.c_uint,
      C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_check_edges_plain", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
      C.POINTER(EdgeParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_edges_workspace_bytes", C.c_size_t, [C.c_int]),
    ("ps_check_edges", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
      C.POINTER(EdgeParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
      C.c_size_t, C.c_void_p]),
    ("ps_check_edges_static", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
      C.POINTER(EdgeParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_traj_cost", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_int, C.c_int,
      C.POINTER(CostParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_rollout_costs", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_int, C.c_int,
      C.POINTER(CostParams), C.c_int, C.c_void_p, C.c_void_p]),
    ("ps_edges_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("ps_edge_bridge_create", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("ps_edge_bridge_set_scene", C.c_int, [C.c_void_p, C.POINTER(SceneView)]),
    ("ps_edge_bridge_evaluate", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(EdgeParams), C.c_void_p, C.c_void_p,
      C.c_void_p]),
    ("ps_edge_bridge_submit", C.c_int,
     [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(EdgeParams)]),
    ("ps_edge_bridge_wait", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_edge_bridge_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("ps_edge_bridge_host_inputs", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    ("ps_edge_bridge_destroy", C.c_int, [C.c_void_p]),
    ("ps_batch_create", C.c_int, [C.c_void_p, C.POINTER(BatchLimits), C.POINTER(C.c_void_p)]),
    ("ps_batch_destroy", C.c_int, [C.c_void_p]),
    ("ps_batch_clear", C.c_int, [C.c_void_p]),
    ("ps_batch_add_edges", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("ps_batch_add_trajectory", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ps_batch_add_rollouts", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    ("ps_batch_launch", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.POINTER(EdgeParams), C.POINTER(CostParams), C.c_void_p]),
    ("ps_batch_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("ps_batch_set_shape", C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
    ("ps_batch_tune", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.POINTER(EdgeParams), C.POINTER(CostParams),
      C.POINTER(BatchTuning)]),
    ("ps_chomp_workspace_bytes", C.c_size_t, [C.c_void_p, C.c_int, C.c_int]),
    ("ps_chomp_optimize", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_int, C.c_int, C.POINTER(ChompParams),
      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("ps_stomp_workspace_bytes", C.c_size_t, [C.c_void_p, C.c_int, C.c_int, C.POINTER(StompParams)]),
    ("ps_stomp_workspace_layout", C.c_int,
     [C.c_void_p, C.c_int, C.c_int, C.POINTER(StompParams), C.POINTER(StompLayout)]),
    ("ps_stomp_optimize", C.c_int,
     [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_int, C.c_int, C.POINTER(StompParams),
      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("ps_fk_spheres", C.c_int,
     [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("ps_probe_fp32_peak", C.c_int, [C.POINTER(C.c_double), C.c_void_p]),
    ("ps_set_stats", C.c_int, [C.c_void_p]),
    ("ps_set_timing_events", C.c_int, [C.c_void_p, C.c_void_p]),
]

EXPORTED_SYMBOLS = [name for name, _, _ in _SIGNATURES]

_lib = None


def load(path: os.PathLike | None = None):
    """Load the CUDA library once and bind every symbol. Raises if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.is_file():
        raise ImportError(
            f"prismplan_b200 CUDA library not found at {p}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` or "
            "`make -C prismplan_b200/csrc`")
    lib = C.CDLL(str(p))
    for name, restype, argtypes in _SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if path is None:
        _lib = lib
    return lib


def check(status: int) -> None:
    if status != PS_OK:
        msg = load().ps_last_error()
        raise PrismError(status, msg.decode() if msg else "")


def stream_handle(stream) -> int | None:
    """cudaStream_t of a torch.cuda.Stream (or None for the current stream)."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) or None
